// BLAST tabular output (output.rs, hsp.rs:84-241) of the drop-in command
// line.  (The blastx front end, translate.rs, runs on the device:
// drg_translate_reads.)
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "drgpu.h"
#include "seqio.h"

namespace drg {
namespace host {

// ---- output.rs -----------------------------------------------------------------
enum Field : int {
  kQSeqId, kQLen, kSSeqId, kSLen, kQStart, kQEnd, kSStart, kSEnd, kQSeq, kSSeq, kEValue, kBitScore, kScore,
  kLength, kPIdent, kNIdent, kMismatch, kPositive, kGapOpen, kGaps, kPPos, kQFrame, kQCovHsp, kSCovHsp, kCigar,
  kBTop, kQTitle, kSTitle, kFullSSeq, kQSeqTranslated, kQStrand
};
// output.rs:116-135; throws std::runtime_error with the reference's message.
std::vector<Field> parse_outfmt_tokens(const std::vector<std::string>& tokens);
std::string format_double(double x);  // output.rs:235-241 (DIAMOND format_double)
std::string format_evalue(double e);  // output.rs:244-250 (Rust "{:.2e}")

struct QueryView {
  const std::string* id;
  const std::string* header;
  const uint8_t* letters;  // letters of the frame the HSP belongs to
  size_t frame_len;
  size_t dna_len;          // nucleotides (blastx) or residues (blastp)
  bool translated;
};
// One tab-separated row (without the newline), output.rs:150-223.
std::string tabular_row(const drg_hsp& h, const uint32_t* ops, const QueryView& q, const DbFile& db,
                        const std::vector<Field>& fields);

}  // namespace host
}  // namespace drg
