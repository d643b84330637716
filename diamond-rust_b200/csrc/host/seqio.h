// Host-side sequence I/O of the drop-in command line: residue encoding
// (alphabet.rs), FASTA reading (io.rs) and the DRDMND01 database file
// (db.rs).  The file format must stay byte-compatible with the reference so
// that databases built by either tool open in the other.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace drg {
namespace host {

constexpr int kAaCount = 25;
constexpr uint8_t kXLetter = 23;
constexpr uint8_t kStopLetter = 24;

uint8_t encode_letter(uint8_t c);                       // alphabet.rs:24-57
std::vector<uint8_t> encode_residues(const std::string& raw);  // alphabet.rs:59-68
char decode_letter(uint8_t l);                          // alphabet.rs:71-73
std::string decode_residues(const uint8_t* l, size_t n);
std::string header_id(const std::string& header);       // alphabet.rs:92-98

struct FastaRecord {
  std::string header, id, raw;  // raw: upper case, layout characters removed
};
// io.rs:40-97; throws std::runtime_error with the reference's message.
std::vector<FastaRecord> parse_fasta_text(const std::string& data);
std::vector<FastaRecord> read_fasta_file(const std::string& path);  // io.rs:30-38

// The database file (db.rs:1-15 layout, little-endian).
struct DbFile {
  std::string path;
  std::vector<uint8_t> data;
  uint64_t n = 0, letters = 0;
  uint64_t seq_off_start = 0, def_off_start = 0, letters_start = 0, defs_start = 0;
  bool protein = true;
  uint64_t seq_offset(uint64_t i) const;
  uint64_t def_offset(uint64_t i) const;
  const uint8_t* seq(uint64_t i) const { return data.data() + letters_start + seq_offset(i); }
  uint64_t seq_len(uint64_t i) const { return seq_offset(i + 1) - seq_offset(i); }
  std::string header(uint64_t i) const;
  std::string id(uint64_t i) const { return header_id(header(i)); }
  std::string report() const;  // db.rs:281-289
};
std::string db_path_with_extension(const std::string& p);  // db.rs:40-48
DbFile open_db(const std::string& path);                   // db.rs:172-225 (throws)
struct DbBuildResult {
  uint64_t sequences = 0, letters = 0;
};
DbBuildResult build_db(const std::string& fasta, const std::string& out_path);  // db.rs:59-160 (throws)
std::string fmt_count(uint64_t n);                                               // db.rs:298-308

}  // namespace host
}  // namespace drg
