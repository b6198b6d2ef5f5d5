// vd_text.cpp -- the generator text format of Tessellation::import_generators
// and Tessellation::read_generators (tessellation.rs:126-171), parsed on the
// host with the reference's rules:
//   * lines end at '\n' (a trailing '\r' is whitespace to what follows);
//   * a line is split at Unicode White_Space (Rust's char::is_whitespace), and
//     a line with no token is skipped;
//   * the first token (the id) is ignored; each of the next three tokens is
//     read as Rust's `str::parse::<f64>` reads it, and a missing or unparsable
//     one is 0.0;
//   * the text must be UTF-8 (a Rust &str is; BufRead::lines fails on a file
//     that is not).
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "vd_internal.h"

namespace vd {
namespace {

// One code point from valid UTF-8 at s[i..n); *len gets its byte count, or 0
// when the bytes there are not a well-formed UTF-8 sequence (overlong forms,
// surrogates and values past U+10FFFF included, as Rust's str checks them).
uint32_t utf8_next(const unsigned char* s, size_t i, size_t n, int* len) {
  const unsigned c = s[i];
  *len = 0;
  if (c < 0x80) { *len = 1; return c; }
  int need;
  uint32_t cp, lo = 0x80, hi = 0xBF;
  if (c >= 0xC2 && c <= 0xDF) { need = 1; cp = c & 0x1F; }
  else if (c >= 0xE0 && c <= 0xEF) {
    need = 2; cp = c & 0x0F;
    if (c == 0xE0) lo = 0xA0;        // no overlong 3-byte forms
    else if (c == 0xED) hi = 0x9F;   // no surrogates
  } else if (c >= 0xF0 && c <= 0xF4) {
    need = 3; cp = c & 0x07;
    if (c == 0xF0) lo = 0x90;        // no overlong 4-byte forms
    else if (c == 0xF4) hi = 0x8F;   // nothing past U+10FFFF
  } else {
    return 0;
  }
  if (i + (size_t)need >= n) return 0;
  for (int k = 1; k <= need; ++k) {
    const unsigned b = s[i + k];
    const unsigned l = k == 1 ? lo : 0x80, h = k == 1 ? hi : 0xBF;
    if (b < l || b > h) return 0;
    cp = (cp << 6) | (b & 0x3F);
  }
  *len = need + 1;
  return cp;
}

// Rust's char::is_whitespace: the Unicode White_Space property.
bool is_white(uint32_t c) {
  return (c >= 0x09 && c <= 0x0D) || c == 0x20 || c == 0x85 || c == 0xA0 || c == 0x1680 ||
         (c >= 0x2000 && c <= 0x200A) || c == 0x2028 || c == 0x2029 || c == 0x202F || c == 0x205F ||
         c == 0x3000;
}

bool ieq(const char* s, size_t n, const char* lit) {
  if (std::strlen(lit) != n) return false;
  for (size_t k = 0; k < n; ++k) {
    char c = s[k];
    if (c >= 'A' && c <= 'Z') c = (char)(c - 'A' + 'a');
    if (c != lit[k]) return false;
  }
  return true;
}

bool digit(char c) { return c >= '0' && c <= '9'; }

}  // namespace

// `str::parse::<f64>` (Rust core, dec2flt): the token must match, after
// lower-casing,
//   Sign? ( 'inf' | 'infinity' | 'nan' | Number ),
//   Number = ( Digit+ | Digit+ '.' Digit* | Digit* '.' Digit+ ) ( 'e' Sign? Digit+ )?
// and the value is the correctly rounded double (round half to even), +-inf
// past the largest double and +-0 below the smallest subnormal.  Returns false
// for any other token.
bool parse_f64(const char* s, size_t n, double* out) {
  size_t i = 0;
  bool neg = false;
  if (i < n && (s[i] == '+' || s[i] == '-')) { neg = s[i] == '-'; ++i; }
  const char* b = s + i;
  const size_t m = n - i;
  if (ieq(b, m, "inf") || ieq(b, m, "infinity")) {
    *out = neg ? -std::numeric_limits<double>::infinity() : std::numeric_limits<double>::infinity();
    return true;
  }
  if (ieq(b, m, "nan")) {
    const double q = std::numeric_limits<double>::quiet_NaN();
    *out = neg ? -q : q;
    return true;
  }
  // Number, validated by hand; the decimal exponent of the leading nonzero
  // digit decides overflow against underflow when the value is out of range
  size_t j = i, nint = 0, nfrac = 0;
  long long lead = std::numeric_limits<long long>::min();  // exponent of the first nonzero digit
  while (j < n && digit(s[j])) {
    if (lead == std::numeric_limits<long long>::min() && s[j] != '0') lead = -(long long)nint - 1;
    ++j; ++nint;
  }
  if (lead != std::numeric_limits<long long>::min()) lead += (long long)nint;  // first nonzero at 10^(nint-1-pos)
  if (j < n && s[j] == '.') {
    ++j;
    while (j < n && digit(s[j])) {
      ++nfrac;
      if (lead == std::numeric_limits<long long>::min() && s[j] != '0') lead = -(long long)nfrac;
      ++j;
    }
  }
  if (nint + nfrac == 0) return false;
  long long ex = 0;
  if (j < n && (s[j] == 'e' || s[j] == 'E')) {
    ++j;
    bool eneg = false;
    if (j < n && (s[j] == '+' || s[j] == '-')) { eneg = s[j] == '-'; ++j; }
    size_t nd = 0;
    while (j < n && digit(s[j])) {
      if (ex < 1000000000LL) ex = ex * 10 + (s[j] - '0');
      ++j; ++nd;
    }
    if (nd == 0) return false;
    if (eneg) ex = -ex;
  }
  if (j != n) return false;
  double v = 0.0;
  // from_chars takes no '+'; it reads the same grammar (general format)
  const auto r = std::from_chars(s + i, s + n, v, std::chars_format::general);
  if (r.ec == std::errc::result_out_of_range) {
    // only a nonzero value can be out of range
    const bool big = lead != std::numeric_limits<long long>::min() && lead + ex >= 0;
    v = big ? std::numeric_limits<double>::infinity() : 0.0;
  } else if (r.ec != std::errc() || r.ptr != s + n) {
    return false;
  }
  *out = neg ? -v : v;
  return true;
}

bool parse_generators(const char* text, size_t len, std::vector<double>* xyz, std::string* err) {
  const unsigned char* s = reinterpret_cast<const unsigned char*>(text);
  xyz->clear();
  size_t i = 0;
  // tokens of the current line: [start, end) byte ranges
  std::vector<std::pair<size_t, size_t>> tok;
  while (i <= len) {
    tok.clear();
    size_t start = SIZE_MAX;
    for (;;) {
      if (i == len || s[i] == '\n') {
        if (start != SIZE_MAX) tok.emplace_back(start, i);
        ++i;
        break;
      }
      int l;
      const uint32_t c = utf8_next(s, i, len, &l);
      if (l == 0) {
        *err = "generator text is not valid UTF-8 at byte " + std::to_string(i);
        return false;
      }
      if (is_white(c)) {
        if (start != SIZE_MAX) { tok.emplace_back(start, i); start = SIZE_MAX; }
      } else if (start == SIZE_MAX) {
        start = i;
      }
      i += (size_t)l;
    }
    if (tok.empty()) continue;  // line.trim().is_empty(), or no id
    for (size_t k = 1; k <= 3; ++k) {
      double v = 0.0;
      if (k < tok.size() && !parse_f64(text + tok[k].first, tok[k].second - tok[k].first, &v)) v = 0.0;
      xyz->push_back(v);
    }
  }
  return true;
}

}  // namespace vd

extern "C" int vd_parse_generators(const char* text, size_t len, double* xyz, size_t cap, size_t* n_points) {
  if ((!text && len) || (!xyz && cap) || !n_points) return VD_EINVAL;
  std::vector<double> v;
  std::string err;
  if (!vd::parse_generators(text, len, &v, &err)) {
    vd::set_thread_error(err.c_str());
    return VD_EINVAL;
  }
  *n_points = v.size() / 3;
  if (cap) std::memcpy(xyz, v.data(), std::min(cap, *n_points) * 3 * sizeof(double));
  return VD_OK;
}
