#include "presets.h"

#include <cmath>

namespace drg {

namespace {
// DIAMOND's shape sets per sensitivity (identical strings to the reference).
const char* const kFast[] = {"1101110101101111"};
const char* const kDefault[] = {"111101110111", "111011010010111"};
const char* const kMid[] = {"11110110111",    "1101100111101",    "1110010101111",    "11010101100111",
                            "11101110001011", "1110100100010111", "1101000011010111", "1110011000011011"};
const char* const kSensitive[] = {"1011110111",       "110100100010111",  "11001011111",      "101110001111",
                                  "11011101100001",   "1111010010101",    "111001001001011",  "10101001101011",
                                  "111101010011",     "1111000010000111", "1100011011011",    "1101010000011011",
                                  "1110001010101001", "110011000110011",  "11011010001101",   "1101001100010011"};
const char* const kVerySensitive[] = {
    "11110111",          "11100100111",         "110010101011",        "11010001001011",
    "10101100001101",    "110100100100011",     "1010010100010011",    "1100101000001011",
    "11100000100010101", "11000100010010011",   "11010000001000111",   "110001001000010011",
    "1010001000100001011", "1100010100000010011", "1100100000101000011", "1101000010000001011"};
const char* const kUltra[] = {
    "1111111",          "11101111",         "110011111",        "110110111",        "111111001",
    "1010111011",       "1011110101",       "1111000111",       "10011110011",      "10101101101",
    "10111010101",      "11001010111",      "11001100111",      "11010101101",      "11110001011",
    "100111010011",     "101100110101",     "101110000111",     "110100101011",     "110110001101",
    "111000110011",     "1010001011011",    "1010101000111",    "1010110100011",    "1100100110011",
    "1100101001011",    "1101001100101",    "1101010101001",    "1110001010101",    "1110010010011",
    "10100001101101",   "11000100010111",   "11010000100111",   "11010100110001",   "11101000011001",
    "11110000001101",   "11110100000011",   "101001000001111",  "110000100101011",  "110010010000111",
    "110101100001001",  "110110000010011",  "111001000100011",  "111100000100101",  "1000110010010101",
    "1001000100101101", "1001000110011001", "1010001001001011", "1010001010010011", "1010010001010101",
    "1010010100010011", "1010010101001001", "1010100000101011", "1010100011000101", "1011000010001011",
    "1100010000111001", "1100010010001011", "1100100001001011", "1100100100100011", "1100110000001101",
    "1101000100010011", "1101000110000101", "1110000001010011", "1110100000010101"};

template <size_t N>
std::vector<ShapeCode> build(const char* const (&codes)[N]) {
  std::vector<ShapeCode> v;
  for (size_t i = 0; i < N; ++i) {
    ShapeCode s;
    parse_shape(codes[i], &s);
    v.push_back(s);
  }
  return v;
}

uint8_t letter_code(char c) {
  static const char* syms = "ARNDCQEGHILKMFPSTWYVBJZX*";
  for (int i = 0; i < 25; ++i)
    if (syms[i] == c) return (uint8_t)i;
  if (c == 'U') return 4;
  if (c == 'O') return 11;
  return 23;
}
}  // namespace

bool parse_shape(const std::string& code, ShapeCode* out) {
  ShapeCode s;
  s.code = code;
  for (size_t i = 0; i < code.size(); ++i) {
    if (code[i] == '1') {
      s.positions.push_back((int)i);
      s.span = (int)i + 1;
    } else if (code[i] == '0') {
      s.span = (int)i + 1;
    } else {
      return false;
    }
  }
  if (s.positions.empty()) return false;
  s.weight = (int)s.positions.size();
  *out = s;
  return true;
}

bool known_sensitivity(const std::string& s) {
  return s == "fast" || s == "faster" || s == "default" || s == "mid-sensitive" || s == "sensitive" ||
         s == "more-sensitive" || s == "very-sensitive" || s == "ultra-sensitive";
}

std::vector<ShapeCode> preset_shapes(const std::string& s) {
  if (s == "faster" || s == "fast") return build(kFast);
  if (s == "mid-sensitive") return build(kMid);
  if (s == "sensitive" || s == "more-sensitive") return build(kSensitive);
  if (s == "very-sensitive") return build(kVerySensitive);
  if (s == "ultra-sensitive") return build(kUltra);
  return build(kDefault);
}

ReducedAlphabet reduction_from_groups(const char* groups) {
  ReducedAlphabet r;
  for (int i = 0; i < 25; ++i) r.bucket[i] = 255;
  int b = 0;
  const char* p = groups;
  while (*p) {
    while (*p == ' ') ++p;
    if (!*p) break;
    while (*p && *p != ' ') {
      uint8_t l = letter_code(*p);
      if (l < 20) r.bucket[l] = (uint8_t)b;
      ++p;
    }
    ++b;
  }
  r.size = b;
  return r;
}

ReducedAlphabet reduction_by_id(int id) {
  if (id == 1) return reduction_from_groups("A G P CH ST NDE RQK FWY ILMV");
  if (id == 2) return reduction_from_groups("A R N D C Q E G H I L K M F P S T W Y V");
  return reduction_from_groups("A KR EDNQ C G H ILVM FYW P ST");
}

ReducedAlphabet preset_reduction(const std::string& s) { return reduction_by_id(s == "very-sensitive" ? 1 : 0); }

double preset_seed_cut(const std::string& s) {
  if (s == "faster" || s == "fast") return 0.9;
  if (s == "mid-sensitive" || s == "sensitive" || s == "more-sensitive" || s == "very-sensitive" ||
      s == "ultra-sensitive")
    return 1.0;
  return 0.8;
}

int preset_index_chunks(const std::string& s) {
  return (s == "very-sensitive" || s == "ultra-sensitive") ? 1 : 4;
}

void ln_factorial_table(double out[33]) {
  out[0] = 0.0;
  out[1] = 0.0;
  for (int n = 2; n < 33; ++n) out[n] = out[n - 1] + std::log((double)n);
}

std::vector<std::pair<uint64_t, uint64_t>> split_chunks(uint64_t n, uint64_t parts) {
  std::vector<std::pair<uint64_t, uint64_t>> v;
  if (parts == 0) parts = 1;
  if (n == 0) return v;
  if (parts > n) parts = n;
  uint64_t start = 0;
  for (uint64_t p = 0; p < parts; ++p) {
    uint64_t end = p + 1 == parts ? n : start + n / parts + (p < n % parts ? 1 : 0);
    v.emplace_back(start, end);
    start = end;
  }
  return v;
}

int band_for_length(uint64_t len) {
  static const uint64_t th[7] = {50, 100, 150, 200, 250, 350, 500};
  static const int bw[8] = {12, 16, 30, 30, 30, 40, 64, 64};
  int b = 0;
  for (uint64_t t : th) b += len >= t;
  return bw[b];
}

}  // namespace drg
