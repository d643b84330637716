// blastx front end on the device: six-frame translation, short-ORF masking
// and the drop of frames without a real residue (translate.rs:54-137,
// workflow.rs:112-127).
//
// Layout: reads are the FASTA records' upper-cased bytes back to back with
// u64 offsets.  One thread per (read, frame) translates its frame into a
// scratch buffer at an offset fixed by the frame's length alone
// ((L - offset) / 3 codons), masks the stop-free stretches shorter than the
// read's minimum ORF length in place, and flags the frame when a letter
// below X survives.  The kept frames are then compacted, in (read, frame)
// order, into the target batch layout the search takes.
#include "kernels.h"

namespace drg {

namespace {

constexpr uint8_t kXLetterDev = 23;     // alphabet.rs X_LETTER
constexpr uint8_t kStopLetterDev = 24;  // alphabet.rs STOP_LETTER

// translate.rs:15-23: T/U 0, C 1, A 2, G 3, anything else 4 (lower case too)
__device__ __forceinline__ uint32_t base_of(uint8_t b) {
  switch (b) {
    case 'T': case 't': case 'U': case 'u': return 0;
    case 'C': case 'c': return 1;
    case 'A': case 'a': return 2;
    case 'G': case 'g': return 3;
    default: return 4;
  }
}
// translate.rs:25-45: complement of the upper-case IUPAC codes; other bytes
// (S, W, N, lower case, ...) stay as they are
__device__ __forceinline__ uint8_t complement_of(uint8_t b) {
  switch (b) {
    case 'A': return 'T';
    case 'T': return 'A';
    case 'C': return 'G';
    case 'G': return 'C';
    case 'U': return 'A';
    case 'R': return 'Y';
    case 'Y': return 'R';
    case 'K': return 'M';
    case 'M': return 'K';
    case 'B': return 'V';
    case 'V': return 'B';
    case 'D': return 'H';
    case 'H': return 'D';
    default: return b;
  }
}

// The standard genetic code (TCAG order) as letter codes, built per block
// from the one-letter table: alphabet index of each codon's amino acid.
__device__ __forceinline__ void stage_codons(uint8_t* codon) {
  const char* code = "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG";
  const char* alphabet = "ARNDCQEGHILKMFPSTWYVBJZX*";
  for (int i = threadIdx.x; i < 64; i += blockDim.x) {
    uint8_t v = kXLetterDev;
    for (int k = 0; k < 25; ++k)
      if (alphabet[k] == code[i]) v = (uint8_t)k;
    codon[i] = v;
  }
  __syncthreads();
}

// translate.rs:124-137 min_orf_len, or the caller's value when >= 0
__device__ __forceinline__ uint64_t min_orf_of(uint64_t dna_len, int64_t user) {
  if (user >= 0) return (uint64_t)user;
  return dna_len < 30 ? 1 : (dna_len < 100 ? 20 : 40);
}

__global__ void k_frame_lengths(const uint64_t* __restrict__ nt_off, uint64_t n_reads, uint64_t* __restrict__ len) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i > 6 * n_reads) return;
  if (i == 6 * n_reads) {
    len[i] = 0;  // the scan's total slot
    return;
  }
  const uint64_t L = nt_off[i / 6 + 1] - nt_off[i / 6];
  const uint64_t o = (i % 6) % 3;
  len[i] = L >= o ? (L - o) / 3 : 0;
}

__global__ void k_translate_frames(TranslateArgs a) {
  __shared__ uint8_t codon[64];
  stage_codons(codon);
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i > 6 * a.n_reads) return;
  if (i == 6 * a.n_reads) {  // the scans' total slots
    a.keep[i] = 0;
    a.kept_len[i] = 0;
    return;
  }
  const uint64_t r = i / 6;
  const int f = (int)(i % 6), o = f % 3;
  const uint8_t* nt = a.nt + a.nt_off[r];
  const uint64_t L = a.nt_off[r + 1] - a.nt_off[r];
  uint8_t* out = a.scratch + a.scratch_off[i];
  const uint64_t n = a.scratch_off[i + 1] - a.scratch_off[i];
  for (uint64_t c = 0; c < n; ++c) {
    uint32_t b[3];
    for (int k = 0; k < 3; ++k) {
      const uint64_t p = o + 3 * c + k;  // position in the strand
      b[k] = f < 3 ? base_of(nt[p]) : base_of(complement_of(nt[L - 1 - p]));
    }
    out[c] = (b[0] > 3 || b[1] > 3 || b[2] > 3) ? kXLetterDev : codon[b[0] * 16 + b[1] * 4 + b[2]];
  }
  // translate.rs:98-118: stop-free stretches shorter than min_len become X
  const uint64_t min_len = min_orf_of(L, a.min_orf);
  if (min_len > 1) {
    uint64_t begin = 0;
    for (uint64_t c = 0; c < n; ++c) {
      if (out[c] != kStopLetterDev) continue;
      if (c - begin < min_len)
        for (uint64_t k = begin; k < c; ++k) out[k] = kXLetterDev;
      begin = c + 1;
    }
    if (n - begin < min_len)
      for (uint64_t k = begin; k < n; ++k) out[k] = kXLetterDev;
  }
  // workflow.rs:118: a frame without a letter below X is not searched
  bool real = false;
  for (uint64_t c = 0; c < n && !real; ++c) real = out[c] < kXLetterDev;
  a.keep[i] = real ? 1 : 0;
  a.kept_len[i] = real ? n : 0;
}

__global__ void k_compact_frames(TranslateArgs a) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i > 6 * a.n_reads) return;
  if (i == 6 * a.n_reads) {  // offsets[n_targets] = letters of all kept frames
    a.out_off[a.kept_index[i]] = a.kept_off[i];
    return;
  }
  if (!a.keep[i]) return;
  const uint64_t t = a.kept_index[i];
  const uint64_t n = a.kept_len[i];
  const uint8_t* src = a.scratch + a.scratch_off[i];
  uint8_t* dst = a.out + a.kept_off[i];
  for (uint64_t c = 0; c < n; ++c) dst[c] = src[c];
  a.out_off[t] = a.kept_off[i];
  a.out_query[t] = (uint32_t)(i / 6);
  a.out_frame[t] = (uint8_t)(i % 6);
}

}  // namespace

void launch_frame_lengths(const uint64_t* nt_off, uint64_t n_reads, uint64_t* len, cudaStream_t st) {
  count_launch();
  k_frame_lengths<<<ceil_div(6 * n_reads + 1, 256), 256, 0, st>>>(nt_off, n_reads, len);
  DRG_CUDA(cudaGetLastError());
}

void launch_translate_frames(const TranslateArgs& a, cudaStream_t st) {
  count_launch();
  k_translate_frames<<<ceil_div(6 * a.n_reads + 1, 128), 128, 0, st>>>(a);
  DRG_CUDA(cudaGetLastError());
}

void launch_compact_frames(const TranslateArgs& a, cudaStream_t st) {
  count_launch();
  k_compact_frames<<<ceil_div(6 * a.n_reads + 1, 128), 128, 0, st>>>(a);
  DRG_CUDA(cudaGetLastError());
}

}  // namespace drg
