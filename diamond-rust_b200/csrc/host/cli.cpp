// The drop-in command line: makedb, blastp, blastx, dbinfo (main.rs,
// workflow.rs, cli.rs).  Option names, defaults, error messages, stderr log
// lines and --outfmt 6 rows follow the reference; the search itself is
// drg_search_run + drg_merge_frames on the GPU (there is no CPU path).
#include <array>
#include <cctype>
#include <cerrno>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "drgpu.h"
#include "seqio.h"
#include "tabular.h"

using namespace drg::host;

namespace {

const char* kVersion = "diamond-rust v0.1.0 (drgpu, B200)";

struct CliError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

size_t default_threads() {  // cli.rs:12-16
  const unsigned n = std::thread::hardware_concurrency();
  return n ? n : 1;
}

// "--name=value" / "--name" / "-n"; false for a non-option argument.
bool split_opt(const std::string& arg, std::string* name, bool* has_inline, std::string* inline_value) {
  if (arg.empty() || arg[0] != '-' || arg == "-") return false;
  size_t k = 0;
  while (k < arg.size() && arg[k] == '-') ++k;
  const std::string s = arg.substr(k);
  if (s.empty()) return false;
  const size_t eq = s.find('=');
  *has_inline = eq != std::string::npos;
  *name = *has_inline ? s.substr(0, eq) : s;
  *inline_value = *has_inline ? s.substr(eq + 1) : std::string();
  return true;
}

std::string take(const std::vector<std::string>& a, size_t* i, bool has_inline, const std::string& inl,
                 const std::string& name) {
  if (has_inline) return inl;
  ++*i;
  if (*i >= a.size()) throw CliError("Option --" + name + " requires a value");
  return a[*i];
}

// Rust's str::parse for usize / i32 / f64 (digits only for the integers).
size_t parse_usize(const std::string& t, const std::string& name) {
  const std::string s = !t.empty() && t[0] == '+' ? t.substr(1) : t;
  if (s.empty() || s.find_first_not_of("0123456789") != std::string::npos)
    throw CliError("Invalid value for --" + name + ": \"" + t + "\"");
  errno = 0;
  const unsigned long long v = std::strtoull(s.c_str(), nullptr, 10);
  if (errno) throw CliError("Invalid value for --" + name + ": \"" + t + "\"");
  return (size_t)v;
}
int parse_i32(const std::string& t, const std::string& name) {
  size_t k = (!t.empty() && (t[0] == '-' || t[0] == '+')) ? 1 : 0;
  if (k == t.size() || t.find_first_not_of("0123456789", k) != std::string::npos)
    throw CliError("Invalid value for --" + name + ": \"" + t + "\"");
  const long long v = std::strtoll(t.c_str(), nullptr, 10);
  if (v < INT32_MIN || v > INT32_MAX) throw CliError("Invalid value for --" + name + ": \"" + t + "\"");
  return (int)v;
}
double parse_f64(const std::string& t, const std::string& name) {
  char* end = nullptr;
  const double v = std::strtod(t.c_str(), &end);
  if (t.empty() || end != t.c_str() + t.size() || std::isspace((unsigned char)t[0]))
    throw CliError("Invalid value for --" + name + ": \"" + t + "\"");
  return v;
}

struct BlastArgs {  // cli.rs:20-40
  std::string db, query, out;
  bool has_out = false;
  std::vector<std::string> outfmt;
  double evalue = 0.001;
  size_t max_target_seqs = 25, max_hsps = 1, threads = default_threads();
  long long index_chunks = -1;
  std::string sensitivity = "default", matrix = "BLOSUM62";
  int gap_open = -1, gap_extend = -1;
  long long min_orf = -1;
  bool has_seed_cut = false;
  double seed_cut = 0;
  bool quiet = false, verbose = true;
};

BlastArgs parse_blast(const std::vector<std::string>& a) {  // cli.rs:125-269
  BlastArgs o;
  bool have_db = false, have_q = false;
  static const char* kIgnoredWithValue[] = {
      "query-gencode", "block-size", "tmpdir", "comp-based-stats", "masking", "motif-masking", "soft-masking",
      "algo", "bin", "swipe", "ext", "query-cover", "subject-cover", "id", "query-length", "approx-id", "log",
      "compress", "chunk-size", "load-threads", "minichunk", "freq-sd", "sketch-size", "tile-size", "id2",
      "padding", "narrow-band-cov", "narrow-band-factor", "min-query-len", "seed-freq", "matrix-scan", "max-hsp",
      "xdrop", "gapped-xdrop", "ungapped-evalue", "gapped-filter-evalue", "toppercent", "top", "sequence-split",
      "blastx", "frameshift", "xml", "json"};
  static const char* kIgnoredFlags[] = {"no-unmask", "unal", "header", "no-reorder", "ignore-warnings", "self",
                                        "iterate", "no-auto-append"};
  static const char* kPresets[] = {"fast", "faster", "mid-sensitive", "sensitive", "more-sensitive",
                                   "very-sensitive", "ultra-sensitive"};
  for (size_t i = 0; i < a.size(); ++i) {
    std::string name, inl;
    bool hi = false;
    if (!split_opt(a[i], &name, &hi, &inl)) throw CliError("Unexpected argument: " + a[i]);
    if (name == "db" || name == "d") {
      o.db = take(a, &i, hi, inl, name);
      have_db = true;
    } else if (name == "query" || name == "q") {
      o.query = take(a, &i, hi, inl, name);
      have_q = true;
    } else if (name == "out" || name == "o") {
      o.out = take(a, &i, hi, inl, name);
      o.has_out = true;
    } else if (name == "outfmt" || name == "f") {
      o.outfmt.push_back(take(a, &i, hi, inl, name));
      while (i + 1 < a.size() && (a[i + 1].empty() || a[i + 1][0] != '-')) o.outfmt.push_back(a[++i]);
    } else if (name == "evalue" || name == "e") {
      o.evalue = parse_f64(take(a, &i, hi, inl, name), name);
    } else if (name == "max-target-seqs" || name == "k") {
      o.max_target_seqs = parse_usize(take(a, &i, hi, inl, name), name);
    } else if (name == "max-hsps") {
      o.max_hsps = parse_usize(take(a, &i, hi, inl, name), name);
    } else if (name == "threads" || name == "p") {
      o.threads = parse_usize(take(a, &i, hi, inl, name), name);
    } else if (name == "index-chunks") {
      o.index_chunks = (long long)parse_usize(take(a, &i, hi, inl, name), name);
    } else if (name == "matrix") {
      o.matrix = take(a, &i, hi, inl, name);
    } else if (name == "gapopen") {
      o.gap_open = parse_i32(take(a, &i, hi, inl, name), name);
    } else if (name == "gapextend") {
      o.gap_extend = parse_i32(take(a, &i, hi, inl, name), name);
    } else if (name == "min-orf" || name == "l") {
      o.min_orf = (long long)parse_usize(take(a, &i, hi, inl, name), name);
    } else if (name == "seed-cut") {
      o.seed_cut = parse_f64(take(a, &i, hi, inl, name), name);
      o.has_seed_cut = true;
    } else if (name == "quiet") {
      o.quiet = true;
    } else if (name == "verbose") {
      o.verbose = true;
    } else {
      bool done = false;
      for (const char* p : kPresets)
        if (name == p) {
          o.sensitivity = p;
          done = true;
        }
      for (const char* p : kIgnoredFlags)
        if (name == p) done = true;
      for (const char* p : kIgnoredWithValue)
        if (name == p) {
          done = true;
          if (!hi && i + 1 < a.size() && (a[i + 1].empty() || a[i + 1][0] != '-') && name != "swipe" &&
              name != "xml" && name != "json")
            ++i;
        }
      if (!done) throw CliError("Unknown option: --" + name);
    }
  }
  if (!have_db) throw CliError("Missing option: --db");
  if (!have_q) throw CliError("Missing option: --query");
  if (o.max_target_seqs < 1) o.max_target_seqs = 1;
  if (o.max_hsps < 1) o.max_hsps = 1;
  if (o.threads < 1) o.threads = 1;
  return o;
}

std::string fmt_seconds(double s) {
  char b[64];
  std::snprintf(b, sizeof b, "%.3f", s);
  return b;
}

int cmd_makedb(const std::vector<std::string>& a) {  // workflow.rs:42-60, cli.rs:88-123
  std::string in, out;
  bool have_in = false, have_out = false, no_auto_append = false, quiet = false;
  for (size_t i = 0; i < a.size(); ++i) {
    std::string name, inl;
    bool hi = false;
    if (!split_opt(a[i], &name, &hi, &inl)) throw CliError("Unexpected argument: " + a[i]);
    if (name == "in" || name == "i") {
      in = take(a, &i, hi, inl, name);
      have_in = true;
    } else if (name == "db" || name == "d") {
      out = take(a, &i, hi, inl, name);
      have_out = true;
    } else if (name == "threads" || name == "p") {
      parse_usize(take(a, &i, hi, inl, name), name);
    } else if (name == "no-auto-append") {
      no_auto_append = true;
    } else if (name == "quiet") {
      quiet = true;
    } else if (name == "verbose") {
    } else if (name == "compress" || name == "compression") {
      take(a, &i, hi, inl, name);
    } else {
      throw CliError("Unknown option: --" + name);
    }
  }
  if (!have_in) throw CliError("Missing option: --in");
  if (!have_out) throw CliError("Missing option: --db");
  const std::string path = no_auto_append ? out : db_path_with_extension(out);
  if (!quiet) std::cerr << kVersion << "\n";
  const auto t0 = std::chrono::steady_clock::now();
  const DbBuildResult r = build_db(in, path);
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (!quiet) {
    std::cerr << "Database: " << path << "\n";
    std::cerr << "Sequences: " << r.sequences << "\n";
    std::cerr << "Letters: " << fmt_count(r.letters) << "\n";
    std::cerr << "Total time = " << fmt_seconds(s) << "s\n";
  }
  return 0;
}

int cmd_dbinfo(const std::vector<std::string>& a) {  // workflow.rs:62-96
  std::string path;
  bool have = false;
  for (size_t i = 0; i < a.size(); ++i) {
    const std::string& arg = a[i];
    std::string rest;
    if (arg.rfind("--", 0) == 0) rest = arg.substr(2);
    else if (arg.rfind("-", 0) == 0) rest = arg.substr(1);
    else throw CliError("Unexpected argument: " + arg);
    const size_t eq = rest.find('=');
    const std::string name = eq == std::string::npos ? rest : rest.substr(0, eq);
    if (name == "db" || name == "d") {
      if (eq != std::string::npos) {
        path = rest.substr(eq + 1);
      } else {
        if (++i >= a.size()) throw CliError("Option --db requires a value");
        path = a[i];
      }
      have = true;
    } else {
      throw CliError("Unknown option: --" + name);
    }
  }
  if (!have) throw CliError("Missing option: --db");
  std::cout << open_db(path).report() << "\n";
  return 0;
}

void check(drg_ctx* ctx, int rc) {
  if (rc == DRG_OK) return;
  const char* msg = ctx ? drg_last_error(ctx) : "";
  if (rc == DRG_ERR_NODEVICE) throw std::runtime_error("no CUDA device: drgpu has no CPU search path");
  throw std::runtime_error(std::string("GPU search failed: ") + msg);
}

int cmd_blast(const std::vector<std::string>& a, bool translated) {  // workflow.rs:98-204
  const BlastArgs o = parse_blast(a);
  if (o.verbose && !o.quiet) std::cerr << kVersion << "\n";
  const auto t0 = std::chrono::steady_clock::now();
  const DbFile db = open_db(o.db);
  const auto records = read_fasta_file(o.query);
  {  // matrix and gap costs are checked before the search (matrix.rs:42-70)
    double e = 0, b = 0;
    if (drg_matrix_evalue(o.matrix.c_str(), o.gap_open, o.gap_extend, 1, 1, 1, 1, &e, &b) != DRG_OK)
      throw std::runtime_error("unsupported matrix or gap costs: " + o.matrix + " " + std::to_string(o.gap_open) +
                               "/" + std::to_string(o.gap_extend));
  }
  drg_ctx* ctx = nullptr;
  check(nullptr, drg_ctx_create(0, &ctx));
  struct CtxGuard {
    drg_ctx*& c;
    ~CtxGuard() {
      if (c) drg_ctx_destroy(c);
    }
  } ctx_guard{ctx};
  const uint8_t empty = 0;
  // targets: translated frames (blastx, on the GPU) or encoded residues (blastp)
  std::vector<std::vector<uint8_t>> t_letters;
  std::vector<uint32_t> t_query;
  std::vector<uint8_t> t_frame;
  std::vector<std::array<long long, 6>> target_of(records.size());
  for (auto& t : target_of) t.fill(-1);
  if (translated) {  // workflow.rs:112-127
    std::vector<uint8_t> nt;
    std::vector<uint64_t> no(1, 0);
    for (const auto& r : records) {
      nt.insert(nt.end(), r.raw.begin(), r.raw.end());
      no.push_back(nt.size());
    }
    uint8_t *L = nullptr, *F = nullptr;
    uint64_t* O = nullptr;
    uint32_t* Q = nullptr;
    uint64_t n = 0;
    check(ctx, drg_translate_reads(ctx, nt.empty() ? &empty : nt.data(), no.data(), records.size(), o.min_orf, &L,
                                   &O, &Q, &F, &n));
    for (uint64_t t = 0; t < n; ++t) {
      target_of[Q[t]][F[t]] = (long long)t;
      t_letters.emplace_back(L + O[t], L + O[t + 1]);
      t_query.push_back(Q[t]);
      t_frame.push_back(F[t]);
    }
    drg_free(L);
    drg_free(O);
    drg_free(Q);
    drg_free(F);
  } else {
    for (size_t qi = 0; qi < records.size(); ++qi) {
      auto l = encode_residues(records[qi].raw);
      if (l.empty()) continue;
      target_of[qi][0] = (long long)t_letters.size();
      t_letters.push_back(std::move(l));
      t_query.push_back((uint32_t)qi);
      t_frame.push_back(0);
    }
  }
  std::vector<uint8_t> tl;
  std::vector<uint64_t> to(1, 0);
  for (const auto& l : t_letters) {
    tl.insert(tl.end(), l.begin(), l.end());
    to.push_back(tl.size());
  }
  std::vector<uint64_t> dbo(db.n + 1);
  for (uint64_t i = 0; i <= db.n; ++i) dbo[i] = db.seq_offset(i);
  drg_search_config cfg{};
  cfg.matrix = o.matrix.c_str();
  cfg.gap_open = o.gap_open;
  cfg.gap_extend = o.gap_extend;
  cfg.evalue = o.evalue;
  cfg.max_target_seqs = (uint32_t)o.max_target_seqs;
  cfg.max_hsps = (uint32_t)o.max_hsps;
  cfg.sensitivity = o.sensitivity.c_str();
  cfg.index_chunks = o.index_chunks < 0 ? -1 : (int32_t)o.index_chunks;
  cfg.has_seed_cut = o.has_seed_cut;
  cfg.seed_cut = o.seed_cut;
  cfg.threads = (uint32_t)o.threads;
  drg_result res{};
  const uint8_t* dl = db.data.data() + db.letters_start;
  const int rc = drg_search_run(ctx, db.letters ? dl : &empty, dbo.data(), db.n, tl.empty() ? &empty : tl.data(),
                                to.data(), t_query.data(), t_frame.data(), t_letters.size(), &cfg, &res);
  if (rc != DRG_OK) throw std::runtime_error("GPU search failed: " + std::string(drg_last_error(ctx)));
  drg_ctx_destroy(ctx);
  ctx = nullptr;
  if (drg_merge_frames(&res, records.size(), t_query.data(), o.max_hsps, o.max_target_seqs) != DRG_OK) {
    drg_result_free(&res);
    throw std::runtime_error("merge_frames failed");
  }
  const auto fields = parse_outfmt_tokens(o.outfmt);
  std::ofstream file;
  if (o.has_out) {
    file.open(o.out, std::ios::binary | std::ios::trunc);
    if (!file) {
      drg_result_free(&res);
      throw std::runtime_error("cannot create " + o.out);
    }
  }
  std::ostream& sink = o.has_out ? static_cast<std::ostream&>(file) : std::cout;
  std::string buf;
  size_t reported = 0, queries_hit = 0;
  for (size_t qi = 0; qi < records.size(); ++qi) {
    const uint64_t lo = res.target_offsets[qi], hi = res.target_offsets[qi + 1];
    if (lo == hi) continue;
    ++queries_hit;
    for (uint64_t k = lo; k < hi; ++k) {
      const drg_hsp& h = res.hsps[k];
      const long long ti = h.frame < 6 ? target_of[qi][h.frame] : -1;
      if (ti < 0) continue;
      QueryView qv{&records[qi].id, &records[qi].header, t_letters[ti].data(), t_letters[ti].size(),
                   records[qi].raw.size(), translated};
      buf += tabular_row(h, res.ops + h.ops_offset, qv, db, fields);
      buf.push_back('\n');
      ++reported;
      if (buf.size() > (1u << 20)) {
        sink << buf;
        buf.clear();
      }
    }
  }
  sink << buf;
  sink.flush();
  drg_result_free(&res);
  if (!o.quiet) {
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cerr << "Total time = " << fmt_seconds(s) << "s\n";
    std::cerr << "Reported " << reported << " pairwise alignments, " << reported << " HSPs.\n";
    std::cerr << queries_hit << " queries aligned.\n";
  }
  return 0;
}

std::string usage_text() {
  return std::string(kVersion) +
         " — a B200 drop-in for the diamond-rust search path\n\n"
         "Usage:\n"
         "  drgpu makedb --in <FASTA> --db <DB> [options]\n"
         "  drgpu blastp --db <DB> --query <FASTA> [options]\n"
         "  drgpu blastx --db <DB> --query <FASTA> [options]\n"
         "  drgpu dbinfo --db <DB>\n\n"
         "Options:\n"
         "  -o, --out <FILE>          output file (default: stdout)\n"
         "  -f, --outfmt <FORMAT>     output format: 6 [field ...] (default: 6)\n"
         "  -e, --evalue <VALUE>      maximum E-value to report (default: 0.001)\n"
         "  -k, --max-target-seqs <N> maximum number of target sequences (default: 25)\n"
         "      --max-hsps <N>        maximum number of HSPs per target (default: 1)\n"
         "  -p, --threads <N>         host threads (default: all cores)\n"
         "      --index-chunks <N>    database chunks indexed at a time (default: preset specific)\n"
         "      --matrix <NAME>       scoring matrix (default: BLOSUM62)\n"
         "      --gapopen <N>         gap open penalty (default: matrix specific)\n"
         "      --gapextend <N>       gap extension penalty (default: matrix specific)\n"
         "  -l, --min-orf <N>         minimum ORF length for blastx\n"
         "      --seed-cut <VALUE>    seed complexity cutoff (default: preset specific)\n"
         "      --fast | --faster | --mid-sensitive | --sensitive\n"
         "      --more-sensitive | --very-sensitive | --ultra-sensitive\n"
         "  -q, --quiet              suppress the progress log\n";
}

}  // namespace

int main(int argc, char** argv) {  // main.rs:3-11
  std::vector<std::string> args(argv + 1, argv + argc);
  if (args.empty()) {
    std::cout << usage_text() << "\n";
    return 1;
  }
  const std::string cmd = args[0];
  const std::vector<std::string> rest(args.begin() + 1, args.end());
  try {
    if (cmd == "version" || cmd == "--version") {
      std::cout << kVersion << "\n";
      return 0;
    }
    if (cmd == "help" || cmd == "--help" || cmd == "-h") {
      std::cout << usage_text() << "\n";
      return 0;
    }
    if (cmd == "makedb") return cmd_makedb(rest);
    if (cmd == "blastp") return cmd_blast(rest, false);
    if (cmd == "blastx") return cmd_blast(rest, true);
    if (cmd == "dbinfo") return cmd_dbinfo(rest);
    std::cerr << "Unknown command: " << cmd << "\n\n";
    std::cout << usage_text() << "\n";
    return 1;
  } catch (const std::exception& e) {
    std::cerr << "Error: " << e.what() << "\n";
    return 1;
  }
}
