// CPU ORACLE -- test infrastructure only (see oracle.h).
// The command line: cli.rs (option parsing) and workflow.rs (makedb, blastp,
// blastx, dbinfo), restated.
#include "oracle.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <thread>

namespace oracle {

namespace {
struct BlastArgs {  // cli.rs:26-46
  std::string db, query, out;
  bool has_out = false;
  std::vector<std::string> outfmt;
  double evalue = 0.001;
  size_t max_target_seqs = 25, max_hsps = 1, threads = 1;
  long index_chunks = -1;
  std::string sensitivity = "default", matrix = "BLOSUM62";
  int gap_open = -1, gap_extend = -1;
  long min_orf = -1;
  double seed_cut = 0;
  bool has_seed_cut = false, quiet = false, verbose = true, translated = false;
};

size_t default_threads() {  // cli.rs:12-16
  unsigned n = std::thread::hardware_concurrency();
  return n ? n : 1;
}

bool split_opt(const std::string& arg, std::string* name, std::string* inl, bool* has_inl) {  // cli.rs:49-61
  if (arg.empty() || arg[0] != '-' || arg == "-") return false;
  size_t b = 0;
  while (b < arg.size() && arg[b] == '-') ++b;
  std::string s = arg.substr(b);
  if (s.empty()) return false;
  size_t eq = s.find('=');
  if (eq == std::string::npos) {
    *name = s;
    *has_inl = false;
  } else {
    *name = s.substr(0, eq);
    *inl = s.substr(eq + 1);
    *has_inl = true;
  }
  return true;
}

struct CliError {
  std::string msg;
};

std::string take_value(const std::vector<std::string>& args, size_t* i, bool has_inl, const std::string& inl,
                       const std::string& name) {
  if (has_inl) return inl;
  *i += 1;
  if (*i >= args.size()) throw CliError{"Option --" + name + " requires a value"};
  return args[*i];
}

size_t parse_usize(const std::string& t, const std::string& name) {
  if (t.empty() || t.find_first_not_of("0123456789") != std::string::npos)
    throw CliError{"Invalid value for --" + name + ": \"" + t + "\""};
  return (size_t)std::stoull(t);
}
int parse_i32(const std::string& t, const std::string& name) {
  try {
    size_t p;
    long v = std::stol(t, &p);
    if (p != t.size()) throw 1;
    return (int)v;
  } catch (...) {
    throw CliError{"Invalid value for --" + name + ": \"" + t + "\""};
  }
}
double parse_f64(const std::string& t, const std::string& name) {
  try {
    size_t p;
    double v = std::stod(t, &p);
    if (p != t.size()) throw 1;
    return v;
  } catch (...) {
    throw CliError{"Invalid value for --" + name + ": \"" + t + "\""};
  }
}

BlastArgs parse_blast(const std::vector<std::string>& args, bool translated) {  // cli.rs:125-269
  BlastArgs a;
  a.translated = translated;
  a.threads = default_threads();
  bool have_db = false, have_q = false;
  static const char* ignored[] = {"query-gencode", "block-size", "tmpdir", "comp-based-stats", "masking",
                                  "motif-masking", "soft-masking", "algo", "bin", "swipe", "ext", "query-cover",
                                  "subject-cover", "id", "query-length", "approx-id", "log", "compress",
                                  "chunk-size", "load-threads", "minichunk", "freq-sd", "sketch-size",
                                  "tile-size", "id2", "padding", "narrow-band-cov", "narrow-band-factor",
                                  "min-query-len", "seed-freq", "matrix-scan", "max-hsp", "xdrop",
                                  "gapped-xdrop", "ungapped-evalue", "gapped-filter-evalue", "toppercent", "top",
                                  "sequence-split", "blastx", "frameshift", "xml", "json"};
  static const char* flags[] = {"no-unmask", "unal", "header", "no-reorder", "ignore-warnings", "self",
                                "iterate", "no-auto-append"};
  for (size_t i = 0; i < args.size(); ++i) {
    std::string name, inl;
    bool has_inl;
    if (!split_opt(args[i], &name, &inl, &has_inl)) throw CliError{"Unexpected argument: " + args[i]};
    if (name == "db" || name == "d") { a.db = take_value(args, &i, has_inl, inl, name); have_db = true; }
    else if (name == "query" || name == "q") { a.query = take_value(args, &i, has_inl, inl, name); have_q = true; }
    else if (name == "out" || name == "o") { a.out = take_value(args, &i, has_inl, inl, name); a.has_out = true; }
    else if (name == "outfmt" || name == "f") {
      a.outfmt.push_back(take_value(args, &i, has_inl, inl, name));
      while (i + 1 < args.size() && !(args[i + 1].size() > 0 && args[i + 1][0] == '-')) a.outfmt.push_back(args[++i]);
    } else if (name == "evalue" || name == "e") a.evalue = parse_f64(take_value(args, &i, has_inl, inl, name), name);
    else if (name == "max-target-seqs" || name == "k") a.max_target_seqs = parse_usize(take_value(args, &i, has_inl, inl, name), name);
    else if (name == "max-hsps") a.max_hsps = parse_usize(take_value(args, &i, has_inl, inl, name), name);
    else if (name == "threads" || name == "p") a.threads = parse_usize(take_value(args, &i, has_inl, inl, name), name);
    else if (name == "index-chunks") a.index_chunks = (long)parse_usize(take_value(args, &i, has_inl, inl, name), name);
    else if (name == "matrix") a.matrix = take_value(args, &i, has_inl, inl, name);
    else if (name == "gapopen") a.gap_open = parse_i32(take_value(args, &i, has_inl, inl, name), name);
    else if (name == "gapextend") a.gap_extend = parse_i32(take_value(args, &i, has_inl, inl, name), name);
    else if (name == "min-orf" || name == "l") a.min_orf = (long)parse_usize(take_value(args, &i, has_inl, inl, name), name);
    else if (name == "seed-cut") { a.seed_cut = parse_f64(take_value(args, &i, has_inl, inl, name), name); a.has_seed_cut = true; }
    else if (name == "fast" || name == "faster" || name == "mid-sensitive" || name == "sensitive" ||
             name == "more-sensitive" || name == "very-sensitive" || name == "ultra-sensitive") a.sensitivity = name;
    else if (name == "quiet") a.quiet = true;
    else if (name == "verbose") a.verbose = true;
    else {
      bool done = false;
      for (const char* ig : ignored)
        if (name == ig) {
          if (!has_inl && i + 1 < args.size() && !(args[i + 1].size() > 0 && args[i + 1][0] == '-'))
            if (!(name == "swipe" || name == "xml" || name == "json")) ++i;
          done = true;
        }
      for (const char* fl : flags)
        if (name == fl) done = true;
      if (!done) throw CliError{"Unknown option: --" + name};
    }
  }
  if (!have_db) throw CliError{"Missing option: --db"};
  if (!have_q) throw CliError{"Missing option: --query"};
  a.max_target_seqs = std::max<size_t>(a.max_target_seqs, 1);
  a.max_hsps = std::max<size_t>(a.max_hsps, 1);
  a.threads = std::max<size_t>(a.threads, 1);
  return a;
}

int cmd_blast(const std::vector<std::string>& args, bool translated) {  // workflow.rs:97-205
  BlastArgs opts = parse_blast(args, translated);
  auto start = std::chrono::steady_clock::now();
  std::string err;
  Database database;
  if (!db_open(opts.db, &database, &err)) throw CliError{err};
  std::vector<Record> records;
  if (!read_fasta(opts.query, &records, &err)) throw CliError{err};
  ScoreMatrix matrix;
  if (!score_matrix_standard(opts.matrix, opts.gap_open, opts.gap_extend, &matrix, &err)) throw CliError{err};
  std::vector<Target> targets;
  std::vector<std::vector<long>> target_of(records.size(), std::vector<long>(6, -1));
  for (size_t qi = 0; qi < records.size(); ++qi) {
    if (translated) {
      size_t min_orf = min_orf_len(records[qi].raw.size(), opts.min_orf);
      auto frames = six_frames(records[qi].raw);
      for (size_t fi = 0; fi < frames.size(); ++fi) {
        mask_short_orfs(frames[fi], min_orf);
        size_t good = 0;
        for (uint8_t l : frames[fi]) good += l < X_LETTER;
        if (good == 0) continue;
        target_of[qi][fi] = (long)targets.size();
        targets.push_back(Target{qi, (uint8_t)fi, std::move(frames[fi])});
      }
    } else {
      auto letters = encode(records[qi].raw);
      if (letters.empty()) continue;
      target_of[qi][0] = (long)targets.size();
      targets.push_back(Target{qi, 0, std::move(letters)});
    }
  }
  SearchConfig cfg;
  cfg.matrix = matrix;
  cfg.evalue = opts.evalue;
  cfg.max_target_seqs = opts.max_target_seqs;
  cfg.max_hsps = opts.max_hsps;
  cfg.sensitivity = opts.sensitivity;
  cfg.threads = opts.threads;
  cfg.index_chunks = opts.index_chunks;
  cfg.seed_cut = opts.seed_cut;
  cfg.has_seed_cut = opts.has_seed_cut;
  RunStats rs;
  auto results = search_run(database, targets, cfg, &rs);
  auto per_query = merge_frames(std::move(results), targets, records.size(), cfg.max_hsps, cfg.max_target_seqs);
  std::vector<int> fields;
  if (!parse_outfmt(opts.outfmt, &fields, &err)) throw CliError{err};
  std::ofstream fout;
  std::ostream* out = &std::cout;
  if (opts.has_out) {
    fout.open(opts.out, std::ios::binary);
    if (!fout) throw CliError{"cannot create " + opts.out};
    out = &fout;
  }
  size_t reported = 0, queries_hit = 0;
  for (size_t qi = 0; qi < per_query.size(); ++qi) {
    if (per_query[qi].empty()) continue;
    ++queries_hit;
    for (const Hsp& h : per_query[qi]) {
      long ti = target_of[qi][h.frame];
      if (ti < 0) continue;
      const auto& letters = targets[(size_t)ti].letters;
      QueryInfo info{records[qi].id, records[qi].header, letters.data(), letters.size(), records[qi].raw.size(),
                     letters.size(), translated};
      *out << tabular_row(h, info, database, fields);
      ++reported;
    }
  }
  out->flush();
  if (!opts.quiet) {
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    fprintf(stderr, "Total time = %.3fs\n", secs);
    fprintf(stderr, "Reported %zu pairwise alignments, %zu HSPs.\n", reported, reported);
    fprintf(stderr, "%zu queries aligned.\n", queries_hit);
    fprintf(stderr, "[oracle] seeds q=%llu r=%llu hits=%llu xdrops=%llu segments=%llu bands=%llu cells=%llu "
                    "seed+join=%.3fs align=%.3fs\n",
            (unsigned long long)rs.query_seeds, (unsigned long long)rs.ref_seeds, (unsigned long long)rs.hits,
            (unsigned long long)rs.xdrops, (unsigned long long)rs.segments, (unsigned long long)rs.bands,
            (unsigned long long)rs.dp_cells, rs.t_seed_join, rs.t_align);
  }
  return 0;
}

// db.rs:298-308 fmt_count: decimal digits grouped by three with commas.
std::string group_thousands(uint64_t v) {
  const std::string d = std::to_string(v);
  std::string out;
  for (size_t i = 0; i < d.size(); ++i) {
    if (i > 0 && (d.size() - i) % 3 == 0) out += ',';
    out += d[i];
  }
  return out;
}

int cmd_makedb(const std::vector<std::string>& args) {  // workflow.rs:42-60 + cli.rs:88-123
  std::string input, output;
  bool have_in = false, have_out = false, no_auto_append = false, quiet = false;
  for (size_t i = 0; i < args.size(); ++i) {
    std::string name, inl;
    bool has_inl;
    if (!split_opt(args[i], &name, &inl, &has_inl)) throw CliError{"Unexpected argument: " + args[i]};
    if (name == "in" || name == "i") { input = take_value(args, &i, has_inl, inl, name); have_in = true; }
    else if (name == "db" || name == "d") { output = take_value(args, &i, has_inl, inl, name); have_out = true; }
    else if (name == "threads" || name == "p") parse_usize(take_value(args, &i, has_inl, inl, name), name);
    else if (name == "no-auto-append") no_auto_append = true;
    else if (name == "quiet") quiet = true;
    else if (name == "verbose") {}
    else if (name == "compress" || name == "compression") take_value(args, &i, has_inl, inl, name);
    else throw CliError{"Unknown option: --" + name};
  }
  if (!have_in) throw CliError{"Missing option: --in"};
  if (!have_out) throw CliError{"Missing option: --db"};
  std::string path = no_auto_append ? output : with_extension(output);
  std::string err;
  size_t n;
  uint64_t letters;
  auto t0 = std::chrono::steady_clock::now();
  if (!db_build(input, path, &err, &n, &letters)) throw CliError{err};
  if (!quiet) {
    fprintf(stderr, "Database: %s\nSequences: %zu\nLetters: %s\nTotal time = %.3fs\n", path.c_str(), n,
            group_thousands(letters).c_str(),
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  }
  return 0;
}
}  // namespace

int cli_main(int argc, char** argv) {
  std::vector<std::string> args(argv + 1, argv + argc);
  try {
    if (args.empty()) {
      printf("oracle: makedb | blastp | blastx | dbinfo\n");
      return 1;
    }
    std::vector<std::string> rest(args.begin() + 1, args.end());
    if (args[0] == "makedb") return cmd_makedb(rest);
    if (args[0] == "blastp") return cmd_blast(rest, false);
    if (args[0] == "blastx") return cmd_blast(rest, true);
    if (args[0] == "dbinfo") {
      std::string path, err;
      for (size_t i = 0; i < rest.size(); ++i) {
        std::string name, inl;
        bool has_inl;
        if (!split_opt(rest[i], &name, &inl, &has_inl)) throw CliError{"Unexpected argument: " + rest[i]};
        if (name == "db" || name == "d") path = take_value(rest, &i, has_inl, inl, name);
        else throw CliError{"Unknown option: --" + name};
      }
      if (path.empty()) throw CliError{"Missing option: --db"};
      Database db;
      if (!db_open(path, &db, &err)) throw CliError{err};
      printf("Database: %s\nSequences: %zu\nLetters: %s\nType: protein\n", db.path.c_str(), db.seq_count,
             group_thousands(db.total_letters).c_str());
      return 0;
    }
    fprintf(stderr, "Unknown command: %s\n", args[0].c_str());
    return 1;
  } catch (const CliError& e) {
    fprintf(stderr, "Error: %s\n", e.msg.c_str());
    return 1;
  } catch (const std::exception& e) {
    fprintf(stderr, "Error: %s\n", e.what());
    return 1;
  }
}

}  // namespace oracle
