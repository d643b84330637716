#include "seqio.h"

#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <sys/stat.h>

namespace drg {
namespace host {

namespace {

const char kSymbols[] = "ARNDCQEGHILKMFPSTWYVBJZX*";

struct LetterTable {
  uint8_t t[256];
  LetterTable() {
    std::memset(t, kXLetter, sizeof t);
    for (int i = 0; i < kAaCount; ++i) {
      const unsigned char c = (unsigned char)kSymbols[i];
      t[c] = (uint8_t)i;
      if (c >= 'A' && c <= 'Z') t[c + 32] = (uint8_t)i;
    }
    // selenocysteine scores as C, pyrrolysine as K
    t[(unsigned char)'U'] = t[(unsigned char)'u'] = 4;
    t[(unsigned char)'O'] = t[(unsigned char)'o'] = 11;
  }
};
const LetterTable kTable;

// u8::is_ascii_whitespace (no vertical tab) and, for trim(), char::is_whitespace on ASCII
bool is_space(unsigned char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f'; }
bool is_trim_space(unsigned char c) { return is_space(c) || c == '\v'; }

uint64_t get64(const std::vector<uint8_t>& d, uint64_t off) {
  uint64_t v = 0;
  std::memcpy(&v, d.data() + off, 8);
  return v;
}
uint32_t get32(const std::vector<uint8_t>& d, uint64_t off) {
  uint32_t v = 0;
  std::memcpy(&v, d.data() + off, 4);
  return v;
}
bool file_exists(const std::string& p) {
  struct stat st;
  return ::stat(p.c_str(), &st) == 0;
}
std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && is_trim_space((unsigned char)s[a])) ++a;
  while (b > a && is_trim_space((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

const char kMagic[8] = {'D', 'R', 'D', 'M', 'N', 'D', '0', '1'};
constexpr uint64_t kHeaderLen = 72;
constexpr uint32_t kVersion = 1, kFlagProtein = 1;

}  // namespace

uint8_t encode_letter(uint8_t c) { return kTable.t[c]; }

std::vector<uint8_t> encode_residues(const std::string& raw) {
  std::vector<uint8_t> out;
  out.reserve(raw.size());
  for (unsigned char c : raw) {
    if (is_space(c) || c == '-' || c == '.') continue;
    out.push_back(kTable.t[c]);
  }
  return out;
}

char decode_letter(uint8_t l) { return kSymbols[l < kAaCount ? l : kAaCount - 1]; }

std::string decode_residues(const uint8_t* l, size_t n) {
  std::string s(n, ' ');
  for (size_t i = 0; i < n; ++i) s[i] = decode_letter(l[i]);
  return s;
}

std::string header_id(const std::string& h) {
  size_t a = 0;
  while (a < h.size() && (h[a] == '>' || h[a] == ' ')) ++a;
  size_t b = a;
  while (b < h.size() && !is_space((unsigned char)h[b])) ++b;
  return h.substr(a, b - a);
}

std::vector<FastaRecord> parse_fasta_text(const std::string& data) {
  std::vector<FastaRecord> out;
  bool have = false, seen_header = false;
  FastaRecord cur;
  auto finish = [&]() {
    size_t b = 0;
    while (b < cur.header.size() && !is_space((unsigned char)cur.header[b])) ++b;
    cur.id = cur.header.substr(0, b);
    if (cur.id.empty()) cur.id = "seq" + std::to_string(cur.raw.size() > 0 ? cur.raw.size() : 1);
    out.push_back(std::move(cur));
    cur = FastaRecord();
  };
  size_t pos = 0;
  while (pos <= data.size()) {
    size_t e = data.find('\n', pos);
    if (e == std::string::npos) e = data.size();
    size_t len = e - pos;
    if (len > 0 && data[pos + len - 1] == '\r') --len;
    const char* line = data.data() + pos;
    if (len > 0 && line[0] == '>') {
      if (have) finish();
      have = seen_header = true;
      cur.header = trim(std::string(line + 1, len - 1));
    } else if (have) {
      for (size_t k = 0; k < len; ++k) {
        const unsigned char c = (unsigned char)line[k];
        if (is_space(c) || c == '-' || c == '.') continue;
        cur.raw.push_back((char)((c >= 'a' && c <= 'z') ? c - 32 : c));
      }
    } else if (len > 0 && line[0] != ';' && line[0] != '#') {
      throw std::runtime_error("malformed FASTA: sequence data found before the first '>' header");
    }
    if (e == data.size()) break;
    pos = e + 1;
  }
  if (have) finish();
  if (!seen_header && !data.empty()) throw std::runtime_error("malformed FASTA: no '>' header found");
  return out;
}

std::vector<FastaRecord> read_fasta_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot read " + path + ": No such file or directory (os error 2)");
  std::stringstream ss;
  ss << f.rdbuf();
  auto recs = parse_fasta_text(ss.str());
  if (recs.empty()) throw std::runtime_error(path + ": no FASTA records found");
  return recs;
}

uint64_t DbFile::seq_offset(uint64_t i) const { return get64(data, seq_off_start + 8 * i); }
uint64_t DbFile::def_offset(uint64_t i) const { return get64(data, def_off_start + 8 * i); }
std::string DbFile::header(uint64_t i) const {
  const uint64_t lo = defs_start + def_offset(i), hi = defs_start + def_offset(i + 1);
  return std::string(reinterpret_cast<const char*>(data.data()) + lo, hi - lo);
}
std::string DbFile::report() const {
  return "Database: " + path + "\nSequences: " + std::to_string(n) + "\nLetters: " + fmt_count(letters) +
         "\nType: protein";
}

std::string db_path_with_extension(const std::string& p) {
  std::string name = p;
  while (name.size() > 1 && name.back() == '/') name.pop_back();
  const size_t slash = name.rfind('/');
  if (slash != std::string::npos) name = name.substr(slash + 1);
  const size_t dot = name.rfind('.');
  const bool has_ext = dot != std::string::npos && dot > 0 && name != "..";
  return has_ext ? p : p + ".dmnd";
}

DbFile open_db(const std::string& path0) {
  std::string path = path0;
  if (!file_exists(path)) {
    const std::string alt = db_path_with_extension(path0);
    if (!file_exists(alt)) throw std::runtime_error("Database file not found: " + path0);
    path = alt;
  }
  DbFile db;
  db.path = path;
  {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read " + path);
    db.data.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  }
  const auto& d = db.data;
  if (d.size() < kHeaderLen) throw std::runtime_error(path + ": not a diamond-rust database (file too short)");
  if (std::memcmp(d.data(), kMagic, 8) != 0)
    throw std::runtime_error(path + ": not a diamond-rust database (bad magic). Build one with `diamond-rust makedb`.");
  const uint32_t version = get32(d, 8);
  if (version != kVersion)
    throw std::runtime_error(path + ": database version " + std::to_string(version) + " is not supported (expected 1)");
  db.protein = (get32(d, 12) & kFlagProtein) != 0;
  db.n = get64(d, 16);
  db.letters = get64(d, 24);
  const uint64_t defs_len = get64(d, 32);
  db.seq_off_start = get64(d, 40);
  db.def_off_start = get64(d, 48);
  db.letters_start = get64(d, 56);
  db.defs_start = get64(d, 64);
  if (db.defs_start + defs_len != d.size()) throw std::runtime_error(path + ": truncated or corrupt database");
  if (db.seq_off_start + 8 * (db.n + 1) > d.size() || db.def_off_start + 8 * (db.n + 1) > d.size())
    throw std::runtime_error(path + ": corrupt offset table");
  return db;
}

DbBuildResult build_db(const std::string& fasta, const std::string& out_path) {
  const auto recs = read_fasta_file(fasta);
  const uint64_t n = recs.size();
  std::vector<std::vector<uint8_t>> enc(n);
  std::vector<uint64_t> so(n + 1), dof(n + 1);
  uint64_t letters = 0, defs = 0;
  for (uint64_t i = 0; i < n; ++i) {
    enc[i] = encode_residues(recs[i].raw);
    if (enc[i].size() > 0xFFFFFFFFull)
      throw std::runtime_error("sequence " + recs[i].id + " is too long for the database format");
    so[i] = letters;
    letters += enc[i].size();
    dof[i] = defs;
    defs += recs[i].header.size();
  }
  so[n] = letters;
  dof[n] = defs;
  const uint64_t seq_off_start = kHeaderLen, def_off_start = seq_off_start + 8 * (n + 1);
  const uint64_t letters_start = def_off_start + 8 * (n + 1), defs_start = letters_start + letters;
  std::ofstream f(out_path, std::ios::binary | std::ios::trunc);
  if (!f) throw std::runtime_error("cannot create " + out_path);
  f.write(kMagic, 8);
  f.write(reinterpret_cast<const char*>(&kVersion), 4);
  f.write(reinterpret_cast<const char*>(&kFlagProtein), 4);
  for (uint64_t v : {n, letters, defs, seq_off_start, def_off_start, letters_start, defs_start})
    f.write(reinterpret_cast<const char*>(&v), 8);
  f.write(reinterpret_cast<const char*>(so.data()), (std::streamsize)(8 * (n + 1)));
  f.write(reinterpret_cast<const char*>(dof.data()), (std::streamsize)(8 * (n + 1)));
  for (const auto& e : enc) f.write(reinterpret_cast<const char*>(e.data()), (std::streamsize)e.size());
  for (const auto& r : recs) f.write(r.header.data(), (std::streamsize)r.header.size());
  if (!f) throw std::runtime_error("cannot write " + out_path);
  return DbBuildResult{n, letters};
}

std::string fmt_count(uint64_t v) {
  const std::string s = std::to_string(v);
  std::string out;
  for (size_t i = 0; i < s.size(); ++i) {
    if (i > 0 && (s.size() - i) % 3 == 0) out.push_back(',');
    out.push_back(s[i]);
  }
  return out;
}

}  // namespace host
}  // namespace drg
