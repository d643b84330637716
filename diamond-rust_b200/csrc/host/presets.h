// Sensitivity presets of the search: seed shapes (shape.rs:78-220), reduced
// alphabets (reduction.rs:48-80), seed-complexity cut (search.rs:55-67) and
// index chunks (search.rs:69-79).  The shape codes and alphabet groupings are
// DIAMOND's published tables and must be identical for the seeds to be.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace drg {

struct ShapeCode {
  std::string code;
  int weight = 0, span = 0;
  std::vector<int> positions;
};

// Parses a 0/1 shape (shape.rs:23-44); false on an invalid code.
bool parse_shape(const std::string& code, ShapeCode* out);

// Shapes of a sensitivity preset; unknown names fall back to "default".
std::vector<ShapeCode> preset_shapes(const std::string& sensitivity);

struct ReducedAlphabet {
  uint8_t bucket[25];  // 255 for letters that cannot seed
  int size;
};
ReducedAlphabet reduction_from_groups(const char* groups);
ReducedAlphabet preset_reduction(const std::string& sensitivity);
ReducedAlphabet reduction_by_id(int id);  // 0 murphy10, 1 diamond9, 2 none

double preset_seed_cut(const std::string& sensitivity);
int preset_index_chunks(const std::string& sensitivity);
bool known_sensitivity(const std::string& s);

// ln n! for n = 0..32, accumulated as t[n] = t[n-1] + ln n (seed.rs:29-38).
void ln_factorial_table(double out[33]);

// seed::chunks (seed.rs:146-164)
std::vector<std::pair<uint64_t, uint64_t>> split_chunks(uint64_t n, uint64_t parts);

// band_for (gapped.rs:27-32)
int band_for_length(uint64_t qlen);

}  // namespace drg
