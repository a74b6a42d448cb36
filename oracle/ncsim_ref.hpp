// CPU ORACLE — test infrastructure only.
//
// A C++ restatement of ncsim's dense `StateVector<C64>` path and the host-side
// pieces it depends on, used as the parity checker for the CUDA engine and as
// the timed CPU baseline.  Nothing in the product library links, includes or
// calls this file; only `tests/`, `__graft_entry__.smoke()` and the
// `cpu_baseline` / `--impl reference` legs of `bench.py` load the oracle.
//
// Parity pins (see tests/test_oracle_*.py):
//   * the known-answer tests of the reference's own test modules, restated:
//     src/state/vector.rs:580-654 (GHZ, Circuit::unitary column),
//     src/state/vector.rs:665-757 (fiber kernel vs the naive O(4^k 2^n) apply,
//     Pauli expectation / apply / project vs the dense Pauli action),
//     src/state/vector.rs:767-800 (Born-rule sampling across blocks),
//     tests/backends.rs:35-226 (StateVector assertions), src/gate.rs:904-984
//     (gate matrices unitary, daggers, monomial composition), src/scalar.rs:428-468;
//   * an independent numpy einsum simulator (tests/golden/numpy_sim.py);
//   * ChaCha against the RFC 8439 block-function test vector.
// Unpinned: bit-level rounding inside the un-vendored `ncalg` complex type
// (Cargo.toml:14, no revision) and the exact output stream of rand 0.8's
// StdRng (no Rust toolchain to produce reference draws); the StdRng here is
// restated from rand_core 0.6 / rand_chacha 0.3 / rand 0.8's published
// algorithms (PCG32 seed expansion, ChaCha12 with a 64-bit block counter,
// 64-word block buffer, 53-bit multiply float conversion, widening-multiply
// range sampling).
//
// Compiled with -O3 -fopenmp -ffp-contract=off: Rust never fuses a*b+c, so the
// restatement does not either.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <omp.h>

namespace ref {

// ---------------------------------------------------------------------------
// errors: src/error.rs:7-42
// ---------------------------------------------------------------------------
enum class ErrKind : int {
  Unsupported = 1,
  QubitOutOfRange = 2,
  Arity = 3,
  DuplicateQubit = 4,
  NotRepresentable = 5,
  ZeroState = 6,
  Parse = 7,
  Invalid = 8,
};

struct SimError : std::runtime_error {
  ErrKind kind;
  SimError(ErrKind k, const std::string& m) : std::runtime_error(m), kind(k) {}
};

// src/error.rs:69-82
inline void check_qubits(const std::vector<size_t>& qubits, size_t n) {
  for (size_t i = 0; i < qubits.size(); ++i) {
    size_t q = qubits[i];
    if (q >= n)
      throw SimError(ErrKind::QubitOutOfRange,
                     "qubit " + std::to_string(q) + " out of range for " + std::to_string(n) + " qubits");
    for (size_t j = 0; j < i; ++j)
      if (qubits[j] == q) throw SimError(ErrKind::DuplicateQubit, "qubit " + std::to_string(q) + " listed twice");
  }
}

// ---------------------------------------------------------------------------
// scalars: src/scalar.rs
// ---------------------------------------------------------------------------
struct C64 {
  double re = 0.0, im = 0.0;
  C64() = default;
  C64(double r, double i) : re(r), im(i) {}
};
inline C64 cadd(C64 a, C64 b) { return {a.re + b.re, a.im + b.im}; }
inline C64 csub(C64 a, C64 b) { return {a.re - b.re, a.im - b.im}; }
inline C64 cmul(C64 a, C64 b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C64 cconj(C64 a) { return {a.re, -a.im}; }
inline C64 cneg(C64 a) { return {-a.re, -a.im}; }
inline bool is_exactly_zero(C64 a) { return a.re == 0.0 && a.im == 0.0; }  // scalar.rs:151
inline bool ceq(C64 a, C64 b) { return a.re == b.re && a.im == b.im; }
inline double norm_sqr(C64 a) { return a.re * a.re + a.im * a.im; }
inline C64 abs_sq(C64 a) { return cmul(a, cconj(a)); }  // scalar.rs:71
inline C64 from_polar(double r, double t) { return {r * std::cos(t), r * std::sin(t)}; }
inline int64_t rem_euclid(int64_t a, int64_t m) {
  int64_t r = a % m;
  return r < 0 ? r + m : r;
}
inline int64_t div_euclid(int64_t a, int64_t m) {
  int64_t q = a / m;
  if (a % m < 0) q += (m > 0 ? -1 : 1);
  return q;
}

// scalar.rs:101-108
inline C64 quarter_turn(int64_t j) {
  switch (rem_euclid(j, 4)) {
    case 0: return {1.0, 0.0};
    case 1: return {0.0, 1.0};
    case 2: return {-1.0, 0.0};
    default: return {0.0, -1.0};
  }
}

// scalar.rs:112-132
inline C64 root_of_unity(int64_t k, uint32_t bits) {
  if (bits > 62) throw SimError(ErrKind::Invalid, "phase bits must be at most 62");
  int64_t m = int64_t(1) << bits;
  k = rem_euclid(k, m);
  if ((4 * k) % m == 0) return quarter_turn(4 * k / m);
  if ((8 * k) % m == 0) {
    const double h = 0.70710678118654752440;  // FRAC_1_SQRT_2
    switch (8 * k / m) {
      case 1: return {h, h};
      case 3: return {-h, h};
      case 5: return {-h, -h};
      default: return {h, -h};
    }
  }
  return from_polar(1.0, 2.0 * 3.14159265358979323846 * double(k) / double(m));
}

// scalar.rs:133-140
inline C64 sqrt2_pow(int64_t k) {
  int64_t half = div_euclid(k, 2);
  double v = std::pow(2.0, double(half));  // powi of 2: exact
  if (rem_euclid(k, 2) == 1) v *= 1.41421356237309504880;  // SQRT_2
  return {v, 0.0};
}

// scalar.rs:54-61
inline C64 i_pow(int64_t k) { return quarter_turn(k); }

// Phasor: scalar.rs:211-376
struct Phasor {
  bool zero = false;
  int32_t sqrt2_power = 0;
  uint64_t phase = 0;
  uint32_t bits = 0;
  static Phasor make(int32_t s2, int64_t phase, uint32_t bits) {  // scalar.rs:234-248
    if (bits > 62) throw SimError(ErrKind::Invalid, "phase bits must be at most 62");
    uint64_t m = uint64_t(1) << bits;
    uint64_t ph = uint64_t(rem_euclid(phase, int64_t(m)));
    while (bits > 0 && ph % 2 == 0) {
      ph /= 2;
      bits -= 1;
    }
    Phasor p;
    p.sqrt2_power = s2;
    p.phase = ph;
    p.bits = bits;
    return p;
  }
  static Phasor one() { return make(0, 0, 0); }
  static Phasor root(int64_t phase, uint32_t bits) { return make(0, phase, bits); }
  static Phasor ipow(int64_t k) { return make(0, k, 2); }
  Phasor mul(const Phasor& o) const {  // scalar.rs:275-295
    if (zero || o.zero) {
      Phasor z;
      z.zero = true;
      return z;
    }
    uint32_t b = std::max(bits, o.bits);
    uint64_t f = (phase << (b - bits)) + (o.phase << (b - o.bits));
    return make(sqrt2_power + o.sqrt2_power, int64_t(f), b);
  }
  bool operator==(const Phasor& o) const {
    if (zero || o.zero) return zero == o.zero;
    return sqrt2_power == o.sqrt2_power && phase == o.phase && bits == o.bits;
  }
};

// scalar.rs:39-52
inline C64 from_phasor(const Phasor& p) {
  if (p.zero) return {0.0, 0.0};
  C64 r = root_of_unity(int64_t(p.phase), p.bits);
  C64 s = sqrt2_pow(p.sqrt2_power);
  return cmul(r, s);
}

// scalar.rs:80-94: pairwise sum, leaves of at most 8
inline C64 pairwise_sum(const C64* items, size_t len) {
  if (len <= 8) {
    C64 acc;
    for (size_t i = 0; i < len; ++i) acc = cadd(acc, items[i]);
    return acc;
  }
  size_t h = len / 2;
  return cadd(pairwise_sum(items, h), pairwise_sum(items + h, len - h));
}

// ---------------------------------------------------------------------------
// StdRng (rand 0.8): ChaCha12 block RNG seeded by PCG32 expansion.
// ---------------------------------------------------------------------------
struct StdRng {
  uint32_t key[8];
  uint64_t counter = 0;  // next block to generate
  uint32_t results[64];
  size_t index = 64;

  static inline uint32_t rotl(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }
  static void block(const uint32_t in[16], uint32_t out[16], int rounds) {
    uint32_t x[16];
    std::memcpy(x, in, sizeof(x));
    auto qr = [&](int a, int b, int c, int d) {
      x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl(x[d], 16);
      x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl(x[b], 12);
      x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl(x[d], 8);
      x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl(x[b], 7);
    };
    for (int r = 0; r < rounds; r += 2) {
      qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
      qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
    }
    for (int i = 0; i < 16; ++i) out[i] = x[i] + in[i];
  }
  // ChaCha state: constants, 8 key words, 64-bit block counter (words 12-13),
  // 64-bit stream id (words 14-15, zero for StdRng).
  void block_at(uint64_t ctr, uint32_t out[16], int rounds = 12) const {
    uint32_t in[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
    for (int i = 0; i < 8; ++i) in[4 + i] = key[i];
    in[12] = uint32_t(ctr);
    in[13] = uint32_t(ctr >> 32);
    in[14] = 0;
    in[15] = 0;
    block(in, out, rounds);
  }
  void refill() {  // four consecutive blocks per refill
    for (int b = 0; b < 4; ++b) block_at(counter + b, results + 16 * b);
    counter += 4;
  }
  static StdRng from_seed(const uint8_t seed[32]) {
    StdRng r;
    for (int i = 0; i < 8; ++i)
      r.key[i] = uint32_t(seed[4 * i]) | (uint32_t(seed[4 * i + 1]) << 8) | (uint32_t(seed[4 * i + 2]) << 16) |
                 (uint32_t(seed[4 * i + 3]) << 24);
    r.counter = 0;
    r.index = 64;
    return r;
  }
  // rand_core 0.6 SeedableRng::seed_from_u64: PCG32 outputs fill the seed.
  static StdRng seed_from_u64(uint64_t state) {
    uint8_t seed[32];
    const uint64_t MUL = 6364136223846793005ull, INC = 11634580027462260723ull;
    for (int i = 0; i < 8; ++i) {
      state = state * MUL + INC;
      uint32_t xorshifted = uint32_t(((state >> 18) ^ state) >> 27);
      uint32_t rot = uint32_t(state >> 59);
      uint32_t x = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
      for (int b = 0; b < 4; ++b) seed[4 * i + b] = uint8_t(x >> (8 * b));
    }
    return from_seed(seed);
  }
  uint32_t next_u32() {
    if (index >= 64) {
      refill();
      index = 0;
    }
    return results[index++];
  }
  uint64_t next_u64() {  // rand_core BlockRng::next_u64
    if (index < 63) {
      uint64_t v = uint64_t(results[index]) | (uint64_t(results[index + 1]) << 32);
      index += 2;
      return v;
    } else if (index >= 64) {
      refill();
      index = 2;
      return uint64_t(results[0]) | (uint64_t(results[1]) << 32);
    } else {
      uint64_t x = results[63];
      refill();
      index = 1;
      return (uint64_t(results[0]) << 32) | x;
    }
  }
  double gen_f64() { return double(next_u64() >> 11) * (1.0 / 9007199254740992.0); }
  bool gen_bool() { return int32_t(next_u32()) < 0; }
  // UniformInt::<u64>::sample_single(0, ub): widening multiply with rejection zone.
  uint64_t gen_range_u64(uint64_t lo, uint64_t hi) {
    if (lo >= hi) throw SimError(ErrKind::Invalid, "gen_range: empty range");
    uint64_t range = hi - lo;
    uint64_t zone = (range << __builtin_clzll(range)) - 1;
    for (;;) {
      uint64_t v = next_u64();
      unsigned __int128 m = (unsigned __int128)v * range;
      uint64_t h = uint64_t(m >> 64), l = uint64_t(m);
      if (l <= zone) return lo + h;
    }
  }
  // UniformInt::<u32>::sample_single(0, ub) (used by slice shuffles for small bounds).
  uint32_t gen_range_u32(uint32_t lo, uint32_t hi) {
    if (lo >= hi) throw SimError(ErrKind::Invalid, "gen_range: empty range");
    uint32_t range = hi - lo;
    uint32_t zone = (range << __builtin_clz(range)) - 1;
    for (;;) {
      uint32_t v = next_u32();
      uint64_t m = uint64_t(v) * range;
      uint32_t h = uint32_t(m >> 32), l = uint32_t(m);
      if (l <= zone) return lo + h;
    }
  }
  // rand 0.8 SliceRandom::shuffle (gen_index uses the u32 sampler below 2^32).
  template <class T>
  void shuffle(std::vector<T>& v) {
    for (size_t i = v.size(); i-- > 1;) {
      size_t j = (i + 1) <= 0xffffffffull ? size_t(gen_range_u32(0, uint32_t(i + 1))) : size_t(gen_range_u64(0, i + 1));
      std::swap(v[i], v[j]);
    }
  }
};

// ---------------------------------------------------------------------------
// Pauli: src/pauli/mod.rs (registers of at most 64 qubits: one word of bits)
// ---------------------------------------------------------------------------
inline int popc(uint64_t v) { return __builtin_popcountll(v); }
inline bool dot(uint64_t a, uint64_t b) { return popc(a & b) & 1; }
inline uint64_t mask_n(size_t n) { return n >= 64 ? ~0ull : ((1ull << n) - 1); }

enum class PauliKind { I, X, Y, Z };

struct Pauli {
  size_t n = 0;
  uint64_t x = 0, z = 0;
  uint8_t phase = 0;  // P = i^phase X^x Z^z

  static Pauli identity(size_t n) { Pauli p; p.n = n; return p; }
  static Pauli make(size_t n, uint64_t x, uint64_t z, uint8_t ph) {  // mod.rs:100-113
    Pauli p;
    p.n = n;
    p.x = x & mask_n(n);
    p.z = z & mask_n(n);
    p.phase = ph & 3;
    return p;
  }
  PauliKind kind(size_t q) const {
    bool bx = (x >> q) & 1, bz = (z >> q) & 1;
    if (bx && bz) return PauliKind::Y;
    if (bx) return PauliKind::X;
    if (bz) return PauliKind::Z;
    return PauliKind::I;
  }
  void set_kind(size_t q, PauliKind k) {  // mod.rs:195-206
    if (q >= n) throw SimError(ErrKind::Invalid, "qubit out of range");
    if (kind(q) == PauliKind::Y) phase = (phase + 3) & 3;
    bool bx = (k == PauliKind::X || k == PauliKind::Y), bz = (k == PauliKind::Z || k == PauliKind::Y);
    x = (x & ~(1ull << q)) | (uint64_t(bx) << q);
    z = (z & ~(1ull << q)) | (uint64_t(bz) << q);
    if (k == PauliKind::Y) phase = (phase + 1) & 3;
  }
  static Pauli single(size_t n, size_t q, PauliKind k) { Pauli p = identity(n); p.set_kind(q, k); return p; }
  static Pauli zq(size_t n, size_t q) { return single(n, q, PauliKind::Z); }
  static Pauli xq(size_t n, size_t q) { return single(n, q, PauliKind::X); }
  static Pauli from_kinds(const std::vector<PauliKind>& ks) {
    Pauli p = identity(ks.size());
    for (size_t q = 0; q < ks.size(); ++q) p.set_kind(q, ks[q]);
    return p;
  }
  bool is_hermitian() const { return ((phase & 1) == 1) == dot(x, z); }  // ops.rs:25-27
  Pauli negated() const { Pauli p = *this; p.phase = (p.phase + 2) & 3; return p; }
  Pauli restrict_to(const std::vector<size_t>& qs) const {  // mod.rs:281-289
    Pauli p = identity(qs.size());
    p.phase = phase;
    for (size_t i = 0; i < qs.size(); ++i) {
      p.x |= ((x >> qs[i]) & 1ull) << i;
      p.z |= ((z >> qs[i]) & 1ull) << i;
    }
    return p;
  }
  Pauli embed(size_t nn, const std::vector<size_t>& qs) const {  // mod.rs:292-301
    if (n != qs.size()) throw SimError(ErrKind::Invalid, "embed: qubit count");
    Pauli p = identity(nn);
    p.phase = phase;
    for (size_t i = 0; i < qs.size(); ++i) {
      p.x |= ((x >> i) & 1ull) << qs[i];
      p.z |= ((z >> i) & 1ull) << qs[i];
    }
    return p;
  }
  void set_raw_bits(size_t q, bool bx, bool bz) {
    x = (x & ~(1ull << q)) | (uint64_t(bx) << q);
    z = (z & ~(1ull << q)) | (uint64_t(bz) << q);
  }
  uint8_t display_phase() const { return uint8_t((phase + 4 - (popc(x & z) % 4)) & 3); }

  // mod.rs:344-414
  static Pauli parse_with(const std::string& s, std::optional<size_t> nreg) {
    auto err = [&](const std::string& m) { return SimError(ErrKind::Parse, "Pauli '" + s + "': " + m); };
    auto trim = [](std::string t) {
      size_t a = t.find_first_not_of(" \t\r\n");
      if (a == std::string::npos) return std::string();
      size_t b = t.find_last_not_of(" \t\r\n");
      return t.substr(a, b - a + 1);
    };
    std::string rest = trim(s);
    uint8_t ph = 0;
    const std::pair<const char*, uint8_t> pres[] = {{"-i", 3}, {"+i", 1}, {"-", 2}, {"+", 0}, {"i", 1}};
    for (auto& pr : pres) {
      std::string pre = pr.first;
      if (rest.compare(0, pre.size(), pre) == 0) {
        std::string r = rest.substr(pre.size());
        size_t a = r.find_first_not_of(" \t\r\n");
        r = a == std::string::npos ? "" : r.substr(a);
        if (!r.empty() && r[0] == '*') r = r.substr(1);
        a = r.find_first_not_of(" \t\r\n");
        r = a == std::string::npos ? "" : r.substr(a);
        ph = pr.second;
        rest = r;
        break;
      }
    }
    bool dense = !rest.empty() && rest.find_first_not_of("IXYZ_") == std::string::npos;
    if (dense) {
      std::vector<PauliKind> ks;
      for (char c : rest)
        ks.push_back(c == 'X' ? PauliKind::X : c == 'Y' ? PauliKind::Y : c == 'Z' ? PauliKind::Z : PauliKind::I);
      Pauli p = from_kinds(ks);
      p.phase = (p.phase + ph) & 3;
      if (nreg && *nreg != ks.size())
        throw err(std::to_string(ks.size()) + " letters for " + std::to_string(*nreg) + " qubits");
      return p;
    }
    std::vector<std::pair<size_t, PauliKind>> sites;
    std::string tok;
    auto flush = [&]() {
      if (tok.empty()) return;
      std::string t = tok;
      tok.clear();
      if (t == "1") return;
      char c = t[0];
      PauliKind k;
      if (c == 'I' || c == '_') k = PauliKind::I;
      else if (c == 'X') k = PauliKind::X;
      else if (c == 'Y') k = PauliKind::Y;
      else if (c == 'Z') k = PauliKind::Z;
      else throw err("token '" + t + "'");
      std::string num = t.substr(1);
      if (num.empty() || num.find_first_not_of("0123456789") != std::string::npos) throw err("token '" + t + "'");
      size_t idx = std::stoull(num);
      for (auto& st : sites)
        if (st.first == idx) throw err("qubit " + std::to_string(idx) + " repeated");
      sites.push_back({idx, k});
    };
    for (char c : rest) {
      if (c == '*' || std::isspace((unsigned char)c)) flush();
      else tok.push_back(c);
    }
    flush();
    size_t n = 0;
    if (nreg) n = *nreg;
    else
      for (auto& st : sites) n = std::max(n, st.first + 1);
    Pauli p = identity(n);
    for (auto& st : sites) {
      if (st.first >= n)
        throw err("qubit " + std::to_string(st.first) + " out of range for " + std::to_string(n) + " qubits");
      p.set_kind(st.first, st.second);
    }
    p.phase = (p.phase + ph) & 3;
    return p;
  }
  static Pauli parse(const std::string& s) { return parse_with(s, std::nullopt); }
  static Pauli from_string(size_t n, const std::string& s) { return parse_with(s, n); }
};

// A Pauli on a register of any width (src/pauli/mod.rs keeps Bits of any
// length): its non-identity letters by qubit (1 = X, 2 = Z, 3 = Y) and the
// phase i^phase in front of the letters.  The same grammar as Pauli::parse.
struct WidePauli {
  size_t n = 0;
  std::vector<std::pair<size_t, uint8_t>> sites;  // ascending qubits
  uint8_t phase = 0;
  bool is_hermitian() const { return (phase & 1) == 0; }
  static WidePauli parse_with(const std::string& s, std::optional<size_t> nreg) {
    auto err = [&](const std::string& m) { return SimError(ErrKind::Parse, "Pauli '" + s + "': " + m); };
    auto trim = [](std::string t) {
      size_t a = t.find_first_not_of(" \t\r\n");
      if (a == std::string::npos) return std::string();
      size_t b = t.find_last_not_of(" \t\r\n");
      return t.substr(a, b - a + 1);
    };
    std::string rest = trim(s);
    WidePauli w;
    const std::pair<const char*, uint8_t> pres[] = {{"-i", 3}, {"+i", 1}, {"-", 2}, {"+", 0}, {"i", 1}};
    for (auto& pr : pres) {
      std::string pre = pr.first;
      if (rest.compare(0, pre.size(), pre) == 0) {
        std::string r = trim(rest.substr(pre.size()));
        if (!r.empty() && r[0] == '*') r = trim(r.substr(1));
        w.phase = pr.second;
        rest = r;
        break;
      }
    }
    auto letter = [](char c) -> uint8_t { return c == 'X' ? 1 : c == 'Z' ? 2 : c == 'Y' ? 3 : 0; };
    bool dense = !rest.empty() && rest.find_first_not_of("IXYZ_") == std::string::npos;
    if (dense) {
      if (nreg && *nreg != rest.size())
        throw err(std::to_string(rest.size()) + " letters for " + std::to_string(*nreg) + " qubits");
      w.n = rest.size();
      for (size_t q = 0; q < rest.size(); ++q)
        if (letter(rest[q])) w.sites.push_back({q, letter(rest[q])});
      return w;
    }
    std::vector<std::pair<size_t, uint8_t>> all;
    std::string tok;
    auto flush = [&]() {
      if (tok.empty()) return;
      std::string t = tok;
      tok.clear();
      if (t == "1") return;
      char c = t[0];
      if (c != 'I' && c != '_' && c != 'X' && c != 'Y' && c != 'Z') throw err("token '" + t + "'");
      std::string num = t.substr(1);
      if (num.empty() || num.find_first_not_of("0123456789") != std::string::npos) throw err("token '" + t + "'");
      size_t idx = std::stoull(num);
      for (auto& st : all)
        if (st.first == idx) throw err("qubit " + std::to_string(idx) + " repeated");
      all.push_back({idx, letter(c)});
    };
    for (char c : rest) {
      if (c == '*' || std::isspace((unsigned char)c)) flush();
      else tok.push_back(c);
    }
    flush();
    if (nreg) w.n = *nreg;
    else
      for (auto& st : all) w.n = std::max(w.n, st.first + 1);
    for (auto& st : all) {
      if (st.first >= w.n)
        throw err("qubit " + std::to_string(st.first) + " out of range for " + std::to_string(w.n) + " qubits");
      if (st.second) w.sites.push_back(st);
    }
    std::sort(w.sites.begin(), w.sites.end());
    return w;
  }
};

// ---------------------------------------------------------------------------
// PhasePoly: src/phasepoly.rs:540-678 (variables fit one word)
// ---------------------------------------------------------------------------
struct PhasePoly {
  size_t n = 0;
  uint32_t bits = 1;
  uint64_t constant = 0;
  std::map<std::vector<uint64_t>, uint64_t> terms;

  PhasePoly() = default;
  PhasePoly(size_t nv, uint32_t b) : n(nv), bits(b) {
    if (b < 1 || b > 32) throw SimError(ErrKind::Invalid, "phase bits must be in 1..=32");
  }
  uint64_t modulus() const { return 1ull << bits; }
  uint64_t reduce(int64_t c) const { return uint64_t(rem_euclid(c, int64_t(modulus()))); }
  void add_constant(int64_t c) { constant = reduce(int64_t(constant) + c); }
  void add_parity_term(int64_t c0, const std::vector<uint64_t>& forms) {  // phasepoly.rs:594-628
    uint64_t c = reduce(c0);
    if (c == 0) return;
    std::vector<uint64_t> key;
    for (uint64_t f : forms) {
      uint64_t g = f & mask_n(n);
      if (g == 0) return;
      key.push_back(g);
    }
    std::sort(key.begin(), key.end());
    key.erase(std::unique(key.begin(), key.end()), key.end());
    if (key.empty()) {
      add_constant(int64_t(c));
      return;
    }
    auto it = terms.find(key);
    if (it != terms.end()) {
      it->second = (it->second + c) % modulus();
      if (it->second == 0) terms.erase(it);
    } else {
      terms[key] = c;
    }
  }
  void add_monomial(int64_t c, const std::vector<size_t>& vars) {
    std::vector<uint64_t> forms;
    for (size_t v : vars) forms.push_back(1ull << v);
    add_parity_term(c, forms);
  }
  void scale(int64_t c) {  // phasepoly.rs:647-657
    uint64_t m = modulus();
    constant = reduce(int64_t(constant) * c);
    std::map<std::vector<uint64_t>, uint64_t> old;
    old.swap(terms);
    for (auto& kv : old) {
      uint64_t w = uint64_t(rem_euclid(int64_t(kv.second) * c, int64_t(m)));
      if (w != 0) terms[kv.first] = w;
    }
  }
  uint64_t eval(uint64_t x) const {  // phasepoly.rs:670-678
    uint64_t acc = constant;
    for (auto& kv : terms) {
      bool all = true;
      for (uint64_t l : kv.first)
        if (!dot(l, x)) { all = false; break; }
      if (all) acc = (acc + kv.second) % modulus();
    }
    return acc;
  }
};

// ---------------------------------------------------------------------------
// MonomialGate: src/gate.rs:30-240
// ---------------------------------------------------------------------------
inline size_t gf2_rank(std::vector<uint64_t> rows, size_t k) {
  size_t rank = 0;
  for (size_t col = 0; col < k && rank < rows.size(); ++col) {
    size_t piv = rank;
    while (piv < rows.size() && !((rows[piv] >> col) & 1)) ++piv;
    if (piv == rows.size()) continue;
    std::swap(rows[piv], rows[rank]);
    for (size_t r = 0; r < rows.size(); ++r)
      if (r != rank && ((rows[r] >> col) & 1)) rows[r] ^= rows[rank];
    ++rank;
  }
  return rank;
}

struct MonomialGate {
  size_t k = 0;
  std::vector<uint64_t> rows;  // row i: the input bits feeding output bit i
  uint64_t shift = 0;
  PhasePoly phase;
  Phasor scalar = Phasor::one();

  static MonomialGate identity(size_t k) {
    MonomialGate g;
    g.k = k;
    for (size_t i = 0; i < k; ++i) g.rows.push_back(1ull << i);
    g.phase = PhasePoly(k, 1);
    return g;
  }
  static MonomialGate make(std::vector<uint64_t> rows, uint64_t shift, PhasePoly phase, Phasor scalar) {
    size_t k = rows.size();
    if (phase.n != k)
      throw SimError(ErrKind::Invalid, "monomial gate: phase polynomial on the wrong number of qubits");
    for (auto& r : rows) r &= mask_n(k);
    if (gf2_rank(rows, k) != k) throw SimError(ErrKind::Invalid, "monomial gate: singular affine map");
    MonomialGate g;
    g.k = k;
    g.rows = rows;
    g.shift = shift & mask_n(k);
    g.phase = phase;
    g.scalar = scalar;
    return g;
  }
  static MonomialGate diagonal(const PhasePoly& p) {
    MonomialGate g = identity(p.n);
    g.phase = p;
    return g;
  }
  static MonomialGate x_string(size_t k, uint64_t a) {
    MonomialGate g = identity(k);
    g.shift = a & mask_n(k);
    return g;
  }
  static MonomialGate permutation(const std::vector<size_t>& perm) {
    std::vector<uint64_t> rows;
    for (size_t j : perm) rows.push_back(1ull << j);
    return make(rows, 0, PhasePoly(perm.size(), 1), Phasor::one());
  }
  static MonomialGate pauli(const Pauli& p) {  // gate.rs:99-108
    MonomialGate g = identity(p.n);
    PhasePoly ph(p.n, 1);
    ph.add_parity_term(1, {p.z});
    g.shift = p.x;
    g.phase = ph;
    g.scalar = Phasor::ipow(p.phase);
    return g;
  }
  // gate.rs:157-169
  std::pair<Phasor, uint64_t> apply_to_basis(uint64_t x) const {
    uint64_t f = phase.eval(x);
    Phasor s = scalar.mul(Phasor::root(int64_t(f), phase.bits));
    uint64_t y = shift;
    for (size_t i = 0; i < rows.size(); ++i)
      if (dot(rows[i], x)) y ^= 1ull << i;
    return {s, y};
  }
  // gate.rs:231-240
  std::vector<C64> matrix() const {
    size_t dim = size_t(1) << k;
    std::vector<C64> m(dim * dim);
    for (size_t x = 0; x < dim; ++x) {
      auto [s, y] = apply_to_basis(x);
      m[y * dim + x] = from_phasor(s);
    }
    return m;
  }
};

// ---------------------------------------------------------------------------
// Gate: src/gate.rs:356-771 (no Clifford tableaux or custom gates: a Clifford
// reaches the dense vector as its dense unitary, i.e. a `Unitary`).
// ---------------------------------------------------------------------------
enum class G {
  I, X, Y, Z, H, S, Sdg, SqrtX, SqrtXdg, SqrtY, SqrtYdg, T, Tdg, Cx, Cy, Cz, Swap, Cs, Csdg, Ccz, Ccx,
  Phase, CPhase, Diagonal, Monomial, PauliG, Rx, Ry, Rz, Unitary
};

struct Gate {
  G g = G::I;
  int64_t pk = 0;     // Phase/CPhase numerator
  uint32_t pbits = 0; // Phase/CPhase bits
  double theta = 0.0;
  PhasePoly poly;     // Diagonal
  MonomialGate mono;  // Monomial
  Pauli pauli;        // Pauli
  size_t uk = 0;      // Unitary arity
  std::vector<C64> umat;

  static Gate named(G g) { Gate x; x.g = g; return x; }
  size_t arity() const {  // gate.rs:447-476
    switch (g) {
      case G::Cx: case G::Cy: case G::Cz: case G::Swap: case G::Cs: case G::Csdg: case G::CPhase: return 2;
      case G::Ccz: case G::Ccx: return 3;
      case G::Diagonal: return poly.n;
      case G::Monomial: return mono.k;
      case G::PauliG: return pauli.n;
      case G::Unitary: return uk;
      default: return 1;
    }
  }
  std::string name() const;

  static MonomialGate mono_phase(size_t k, uint32_t bits, const std::vector<std::pair<int64_t, std::vector<size_t>>>& ts) {
    PhasePoly p(k, bits);
    for (auto& t : ts) p.add_monomial(t.first, t.second);
    return MonomialGate::diagonal(p);
  }
  // gate.rs:519-564
  std::optional<MonomialGate> monomial() const {
    switch (g) {
      case G::I: return MonomialGate::identity(1);
      case G::X: return MonomialGate::x_string(1, 1);
      case G::Y: return MonomialGate::pauli(Pauli::single(1, 0, PauliKind::Y));
      case G::Z: return mono_phase(1, 1, {{1, {0}}});
      case G::S: return mono_phase(1, 2, {{1, {0}}});
      case G::Sdg: return mono_phase(1, 2, {{3, {0}}});
      case G::T: return mono_phase(1, 3, {{1, {0}}});
      case G::Tdg: return mono_phase(1, 3, {{7, {0}}});
      case G::Phase: return mono_phase(1, pbits, {{pk, {0}}});
      case G::CPhase: return mono_phase(2, pbits, {{pk, {0, 1}}});
      case G::Cz: return mono_phase(2, 1, {{1, {0, 1}}});
      case G::Cs: return mono_phase(2, 2, {{1, {0, 1}}});
      case G::Csdg: return mono_phase(2, 2, {{3, {0, 1}}});
      case G::Ccz: return mono_phase(3, 1, {{1, {0, 1, 2}}});
      case G::Cx: return MonomialGate::make({1ull, 3ull}, 0, PhasePoly(2, 1), Phasor::one());
      case G::Cy: {
        PhasePoly p(2, 2);
        p.add_monomial(1, {0});
        p.add_monomial(2, {0, 1});
        return MonomialGate::make({1ull, 3ull}, 0, p, Phasor::one());
      }
      case G::Swap: return MonomialGate::permutation({1, 0});
      case G::Diagonal: return MonomialGate::diagonal(poly);
      case G::Monomial: return mono;
      case G::PauliG: return MonomialGate::pauli(pauli);
      default: return std::nullopt;
    }
  }
  // gate.rs:670-747
  std::optional<std::vector<C64>> matrix() const {
    const C64 half{0.5, 0.0}, i{0.0, 1.0}, one{1.0, 0.0};
    switch (g) {
      case G::H: {
        C64 r = sqrt2_pow(-1);
        return std::vector<C64>{r, r, r, cneg(r)};
      }
      case G::SqrtX: {
        C64 a = cmul(cadd(one, i), half), b = cmul(csub(one, i), half);
        return std::vector<C64>{a, b, b, a};
      }
      case G::SqrtXdg: {
        C64 a = cmul(csub(one, i), half), b = cmul(cadd(one, i), half);
        return std::vector<C64>{a, b, b, a};
      }
      case G::SqrtY: {
        C64 a = cmul(cadd(one, i), half);
        return std::vector<C64>{a, cneg(a), a, a};
      }
      case G::SqrtYdg: {
        C64 a = cmul(csub(one, i), half);
        return std::vector<C64>{a, a, cneg(a), a};
      }
      case G::Ccx: {
        std::vector<C64> m(64);
        for (size_t x = 0; x < 8; ++x) {
          size_t y = (x & 3) == 3 ? (x ^ 4) : x;
          m[y * 8 + x] = one;
        }
        return m;
      }
      case G::Rx: case G::Ry: case G::Rz: {
        double c = std::cos(theta / 2.0), s = std::sin(theta / 2.0);
        C64 z{0.0, 0.0};
        if (g == G::Rx) return std::vector<C64>{{c, 0.0}, {0.0, -s}, {0.0, -s}, {c, 0.0}};
        if (g == G::Ry) return std::vector<C64>{{c, 0.0}, {-s, 0.0}, {s, 0.0}, {c, 0.0}};
        return std::vector<C64>{from_polar(1.0, -theta / 2.0), z, z, from_polar(1.0, theta / 2.0)};
      }
      case G::Unitary: return umat;
      default: {
        auto m = monomial();
        if (!m) return std::nullopt;
        return m->matrix();
      }
    }
  }
  // gate.rs:774-812 (the subset the tests need: daggers of named gates)
  Gate dagger() const {
    Gate d = *this;
    switch (g) {
      case G::S: d.g = G::Sdg; break;
      case G::Sdg: d.g = G::S; break;
      case G::SqrtX: d.g = G::SqrtXdg; break;
      case G::SqrtXdg: d.g = G::SqrtX; break;
      case G::SqrtY: d.g = G::SqrtYdg; break;
      case G::SqrtYdg: d.g = G::SqrtY; break;
      case G::T: d.g = G::Tdg; break;
      case G::Tdg: d.g = G::T; break;
      case G::Cs: d.g = G::Csdg; break;
      case G::Csdg: d.g = G::Cs; break;
      case G::Phase: case G::CPhase: d.pk = -pk; break;
      case G::Diagonal: d.poly.scale(-1); break;
      case G::Rx: case G::Ry: case G::Rz: d.theta = -theta; break;
      case G::Unitary: {
        size_t dim = size_t(1) << uk;
        for (size_t ij = 0; ij < dim * dim; ++ij) d.umat[ij] = cconj(umat[(ij % dim) * dim + ij / dim]);
        break;
      }
      case G::Monomial: case G::PauliG:
        throw SimError(ErrKind::Unsupported, "dagger of a monomial gate is not restated");
      default: break;
    }
    return d;
  }
};

inline std::string fmt_double(double v) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.17g", v);
  return buf;
}

inline std::string Gate::name() const {  // gate.rs:479-515
  switch (g) {
    case G::I: return "I"; case G::X: return "X"; case G::Y: return "Y"; case G::Z: return "Z";
    case G::H: return "H"; case G::S: return "S"; case G::Sdg: return "S_DAG";
    case G::SqrtX: return "SQRT_X"; case G::SqrtXdg: return "SQRT_X_DAG";
    case G::SqrtY: return "SQRT_Y"; case G::SqrtYdg: return "SQRT_Y_DAG";
    case G::T: return "T"; case G::Tdg: return "T_DAG";
    case G::Cx: return "CX"; case G::Cy: return "CY"; case G::Cz: return "CZ"; case G::Swap: return "SWAP";
    case G::Cs: return "CS"; case G::Csdg: return "CS_DAG"; case G::Ccz: return "CCZ"; case G::Ccx: return "CCX";
    case G::Phase: return "PHASE(" + std::to_string(pk) + "," + std::to_string(pbits) + ")";
    case G::CPhase: return "CPHASE(" + std::to_string(pk) + "," + std::to_string(pbits) + ")";
    case G::Rx: return "RX(" + fmt_double(theta) + ")";
    case G::Ry: return "RY(" + fmt_double(theta) + ")";
    case G::Rz: return "RZ(" + fmt_double(theta) + ")";
    case G::Diagonal: return "DIAG";
    case G::Monomial: return "MONOMIAL";
    case G::PauliG: return "PAULI";
    case G::Unitary: return "UNITARY";
  }
  return "?";
}

// ---------------------------------------------------------------------------
// circuits and noise: src/circuit.rs:38-146, 151-237, 459-691
// ---------------------------------------------------------------------------
enum class NoiseKind { XError, YError, ZError, PauliChannel1, Depolarize1, Depolarize2 };
struct Noise {
  NoiseKind kind = NoiseKind::XError;
  double p1 = 0, p2 = 0, p3 = 0;
  size_t arity() const { return kind == NoiseKind::Depolarize2 ? 2 : 1; }
  struct Err { double p; uint8_t x, z; };
  std::vector<Err> errors() const {  // circuit.rs:119-128
    switch (kind) {
      case NoiseKind::XError: return {{p1, 1, 0}};
      case NoiseKind::YError: return {{p1, 1, 1}};
      case NoiseKind::ZError: return {{p1, 0, 1}};
      case NoiseKind::PauliChannel1: return {{p1, 1, 0}, {p2, 1, 1}, {p3, 0, 1}};
      case NoiseKind::Depolarize1: return {{p1 / 3.0, 1, 0}, {p1 / 3.0, 1, 1}, {p1 / 3.0, 0, 1}};
      case NoiseKind::Depolarize2: {
        std::vector<Err> v;
        for (uint8_t k = 1; k < 16; ++k) v.push_back({p1 / 15.0, uint8_t(k & 3), uint8_t(k >> 2)});
        return v;
      }
    }
    return {};
  }
  bool is_valid() const {
    double s = 0;
    for (auto& e : errors()) {
      if (!(e.p >= 0.0 && e.p <= 1.0)) return false;
      s += e.p;
    }
    return s <= 1.0 + 1e-12;
  }
  // circuit.rs:136-146: always one draw
  std::optional<std::pair<uint8_t, uint8_t>> sample(StdRng& rng) const {
    double u = rng.gen_f64();
    for (auto& e : errors()) {
      if (u < e.p) return std::make_pair(e.x, e.z);
      u -= e.p;
    }
    return std::nullopt;
  }
};

enum class OpKind { GateOp, Measure, Reset, NoiseOp, Detector, Observable, Tick };
struct Op {
  OpKind kind = OpKind::Tick;
  Gate gate;
  std::vector<size_t> qubits;
  Pauli pauli;      // measured Pauli (registers of at most 64 qubits)
  WidePauli wide;   // measured Pauli, any register
  size_t qubit = 0;
  Noise noise;
  std::vector<size_t> lookback;  // DETECTOR / OBSERVABLE_INCLUDE rec[-k]
  size_t index = 0;              // OBSERVABLE_INCLUDE(index)
};

struct Circuit {
  size_t n = 0;
  std::vector<Op> ops;
  explicit Circuit(size_t nq = 0) : n(nq) {}
  size_t num_measurements() const {
    size_t m = 0;
    for (auto& o : ops) m += o.kind == OpKind::Measure;
    return m;
  }
  size_t num_gates() const {
    size_t m = 0;
    for (auto& o : ops) m += o.kind == OpKind::GateOp;
    return m;
  }
  void push(const Op& op) {  // circuit.rs:178-229
    switch (op.kind) {
      case OpKind::GateOp:
        check_qubits(op.qubits, n);
        if (op.qubits.size() != op.gate.arity())
          throw SimError(ErrKind::Arity, "gate " + op.gate.name() + " acts on " + std::to_string(op.gate.arity()) +
                                             " qubits, " + std::to_string(op.qubits.size()) + " given");
        break;
      case OpKind::Measure:
        if (op.pauli.n != n || op.wide.n != n) throw SimError(ErrKind::Invalid, "measurement on the wrong register");
        if (!op.pauli.is_hermitian() || !op.wide.is_hermitian())
          throw SimError(ErrKind::Invalid, "measured operator is not Hermitian");
        break;
      case OpKind::Reset: check_qubits({op.qubit}, n); break;
      case OpKind::NoiseOp:
        check_qubits(op.qubits, n);
        if (op.qubits.size() != op.noise.arity()) throw SimError(ErrKind::Arity, "noise arity");
        if (!op.noise.is_valid()) throw SimError(ErrKind::Invalid, "not a probability distribution");
        break;
      default: break;
    }
    ops.push_back(op);
  }
  void gate(const Gate& g, const std::vector<size_t>& qs) {
    Op o;
    o.kind = OpKind::GateOp;
    o.gate = g;
    o.qubits = qs;
    push(o);
  }
  static Circuit parse(const std::string& text);
};

// Extension to the text format (the reference prints DIAG[...] / MONOMIAL[...]
// but does not parse them): `DIAG(bits;const;c:m,m,...;c:m,...) q0 q1 ...`
// with each term `coefficient:parity-mask,...` over the gate's local
// variables, and `MONOMIAL(rows;shift;bits;const;terms...;s2,phase,pbits) q...`.
inline Gate parse_gate_token(const std::string& tok0, const std::vector<std::string>& args, bool& is_gate);

inline std::string upper(std::string s) {
  for (auto& c : s) c = char(std::toupper((unsigned char)c));
  return s;
}

inline std::vector<std::string> split(const std::string& s, char sep) {
  std::vector<std::string> out;
  std::string cur;
  for (char c : s) {
    if (c == sep) {
      out.push_back(cur);
      cur.clear();
    } else cur.push_back(c);
  }
  out.push_back(cur);
  return out;
}

inline std::string trim(const std::string& t) {
  size_t a = t.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return std::string();
  size_t b = t.find_last_not_of(" \t\r\n");
  return t.substr(a, b - a + 1);
}

inline bool parse_i64(const std::string& s, int64_t& v) {
  std::string t = trim(s);
  if (t.empty()) return false;
  char* end = nullptr;
  errno = 0;
  long long x = std::strtoll(t.c_str(), &end, 10);
  if (errno || *end) return false;
  v = x;
  return true;
}
inline bool parse_u64(const std::string& s, uint64_t& v) {
  std::string t = trim(s);
  if (t.empty() || t[0] == '-' || t[0] == '+') return false;
  char* end = nullptr;
  errno = 0;
  unsigned long long x = std::strtoull(t.c_str(), &end, 10);
  if (errno || *end) return false;
  v = x;
  return true;
}
inline bool parse_f64(const std::string& s, double& v) {
  std::string t = trim(s);
  if (t.empty()) return false;
  char* end = nullptr;
  v = std::strtod(t.c_str(), &end);
  return *end == 0;
}

// PhasePoly from `bits;const;c:m,m;c:m` (local masks).
inline PhasePoly parse_poly(size_t nv, const std::vector<std::string>& parts, size_t start) {
  uint64_t bits, cst;
  if (parts.size() < start + 2 || !parse_u64(parts[start], bits) || !parse_u64(parts[start + 1], cst))
    throw SimError(ErrKind::Parse, "phase polynomial needs bits;constant");
  PhasePoly p(nv, uint32_t(bits));
  p.add_constant(int64_t(cst));
  for (size_t i = start + 2; i < parts.size(); ++i) {
    auto ct = split(parts[i], ':');
    int64_t c;
    if (ct.size() != 2 || !parse_i64(ct[0], c)) throw SimError(ErrKind::Parse, "bad term '" + parts[i] + "'");
    std::vector<uint64_t> forms;
    for (auto& m : split(ct[1], ',')) {
      uint64_t v;
      if (!parse_u64(m, v)) throw SimError(ErrKind::Parse, "bad parity '" + m + "'");
      forms.push_back(v);
    }
    p.add_parity_term(c, forms);
  }
  return p;
}

inline Circuit Circuit::parse(const std::string& text) {  // circuit.rs:459-565
  auto err = [](size_t line, const std::string& m) {
    return SimError(ErrKind::Parse, "line " + std::to_string(line + 1) + ": " + m);
  };
  struct PL {
    int kind;  // 0 gate 1 measure-basis 2 mpp 3 reset 4 noise 5 detector 6 observable 7 tick
    Gate g;
    PauliKind pk = PauliKind::Z;
    std::vector<size_t> qs;
    std::vector<std::string> mpp;
    Noise noise;
    std::vector<size_t> recs;
    size_t index = 0;
    size_t ln = 0;
    size_t diag_vars = 0;
  };
  std::vector<std::string> lines = split(text, '\n');
  std::optional<size_t> declared;
  std::vector<PL> parsed;
  size_t max_q = 0;
  for (size_t ln = 0; ln < lines.size(); ++ln) {
    std::string line = trim(split(lines[ln], '#')[0]);
    if (line.empty()) continue;
    std::vector<std::string> toks;
    {
      std::string cur;
      for (char c : line) {
        if (std::isspace((unsigned char)c)) {
          if (!cur.empty()) toks.push_back(cur), cur.clear();
        } else cur.push_back(c);
      }
      if (!cur.empty()) toks.push_back(cur);
    }
    if (upper(toks[0]) == "QUBITS") {
      uint64_t v;
      if (toks.size() < 2 || !parse_u64(toks[1], v)) throw err(ln, "QUBITS n");
      declared = size_t(v);
      continue;
    }
    // parse_args: circuit.rs:579-590
    std::string name;
    std::vector<std::string> args;
    size_t lp = toks[0].find('(');
    if (lp == std::string::npos) name = upper(toks[0]);
    else {
      name = upper(toks[0].substr(0, lp));
      std::string rest = toks[0].substr(lp + 1);
      size_t close = rest.rfind(')');
      if (close == std::string::npos) throw err(ln, "missing ')' in " + toks[0]);
      for (auto& a : split(rest.substr(0, close), ',')) args.push_back(trim(a));
    }
    auto qubits = [&]() {
      std::vector<size_t> qs;
      for (size_t i = 1; i < toks.size(); ++i) {
        uint64_t v;
        if (!parse_u64(toks[i], v)) throw err(ln, "bad qubit '" + toks[i] + "'");
        qs.push_back(size_t(v));
      }
      return qs;
    };
    auto int_arg = [&](size_t i) {
      int64_t v;
      if (i >= args.size() || !parse_i64(args[i], v))
        throw err(ln, name + " needs integer argument " + std::to_string(i + 1));
      return v;
    };
    auto float_arg = [&](size_t i) {
      double v;
      if (i >= args.size() || !parse_f64(args[i], v)) throw err(ln, name + " needs a numeric argument");
      return v;
    };
    PL pl;
    pl.ln = ln;
    pl.kind = 0;
    static const std::map<std::string, G> named = {
        {"I", G::I}, {"X", G::X}, {"Y", G::Y}, {"Z", G::Z}, {"H", G::H}, {"S", G::S}, {"S_DAG", G::Sdg},
        {"SQRT_X", G::SqrtX}, {"SQRT_X_DAG", G::SqrtXdg}, {"SQRT_Y", G::SqrtY}, {"SQRT_Y_DAG", G::SqrtYdg},
        {"T", G::T}, {"T_DAG", G::Tdg}, {"CX", G::Cx}, {"CNOT", G::Cx}, {"CY", G::Cy}, {"CZ", G::Cz},
        {"SWAP", G::Swap}, {"CS", G::Cs}, {"CS_DAG", G::Csdg}, {"CCZ", G::Ccz}, {"CCX", G::Ccx},
        {"TOFFOLI", G::Ccx}};
    auto it = named.find(name);
    if (it != named.end()) {
      pl.g = Gate::named(it->second);
      pl.qs = qubits();
    } else if (name == "PHASE" || name == "CPHASE") {
      pl.g.g = name == "PHASE" ? G::Phase : G::CPhase;
      pl.g.pk = int_arg(0);
      pl.g.pbits = uint32_t(int_arg(1));
      if (pl.g.pbits < 1 || pl.g.pbits > 32) throw err(ln, "phase bits must be in 1..=32");
      pl.qs = qubits();
    } else if (name == "RX" || name == "RY" || name == "RZ") {
      pl.g.g = name == "RX" ? G::Rx : name == "RY" ? G::Ry : G::Rz;
      pl.g.theta = float_arg(0);
      pl.qs = qubits();
    } else if (name == "DIAG") {
      pl.qs = qubits();
      std::string inner = toks[0].substr(lp + 1, toks[0].rfind(')') - lp - 1);
      pl.g.g = G::Diagonal;
      pl.g.poly = parse_poly(pl.qs.size(), split(inner, ';'), 0);
    } else if (name == "MONOMIAL") {
      pl.qs = qubits();
      size_t k = pl.qs.size();
      std::string inner = toks[0].substr(lp + 1, toks[0].rfind(')') - lp - 1);
      auto parts = split(inner, ';');
      if (parts.size() < 5) throw err(ln, "MONOMIAL(rows;shift;bits;const;...;scalar)");
      std::vector<uint64_t> rows;
      for (auto& r : split(parts[0], ',')) {
        uint64_t v;
        if (!parse_u64(r, v)) throw err(ln, "bad row");
        rows.push_back(v);
      }
      uint64_t sh;
      if (!parse_u64(parts[1], sh)) throw err(ln, "bad shift");
      auto sc = split(parts.back(), ',');
      int64_t s2, sp, sb;
      if (sc.size() != 3 || !parse_i64(sc[0], s2) || !parse_i64(sc[1], sp) || !parse_i64(sc[2], sb))
        throw err(ln, "bad scalar");
      std::vector<std::string> pp(parts.begin() + 2, parts.end() - 1);
      PhasePoly poly = parse_poly(k, pp, 0);
      if (rows.size() != k) throw err(ln, "MONOMIAL rows do not match its qubits");
      pl.g.g = G::Monomial;
      pl.g.mono = MonomialGate::make(rows, sh, poly, Phasor::make(int32_t(s2), sp, uint32_t(sb)));
    } else if (name == "M" || name == "MZ" || name == "MX" || name == "MY") {
      pl.kind = 1;
      pl.pk = name == "MX" ? PauliKind::X : name == "MY" ? PauliKind::Y : PauliKind::Z;
      pl.qs = qubits();
    } else if (name == "MPP") {
      pl.kind = 2;
      for (size_t i = 1; i < toks.size(); ++i) {
        WidePauli::parse_with(toks[i], std::nullopt);  // validates
        pl.mpp.push_back(toks[i]);
      }
    } else if (name == "R") {
      pl.kind = 3;
      pl.qs = qubits();
    } else if (name == "DETECTOR" || name == "OBSERVABLE_INCLUDE") {
      for (size_t i = 1; i < toks.size(); ++i) {
        const std::string& t = toks[i];
        uint64_t v;
        if (t.rfind("rec[-", 0) != 0 || t.back() != ']' || !parse_u64(t.substr(5, t.size() - 6), v))
          throw err(ln, "bad target '" + t + "' (expected rec[-k])");
        pl.recs.push_back(size_t(v));
      }
      if (name == "DETECTOR") pl.kind = 5;
      else {
        pl.kind = 6;
        pl.index = size_t(int_arg(0));
      }
    } else if (name == "X_ERROR" || name == "Y_ERROR" || name == "Z_ERROR" || name == "DEPOLARIZE1" ||
               name == "DEPOLARIZE2") {
      pl.kind = 4;
      pl.noise.kind = name == "X_ERROR" ? NoiseKind::XError : name == "Y_ERROR" ? NoiseKind::YError
                    : name == "Z_ERROR" ? NoiseKind::ZError : name == "DEPOLARIZE1" ? NoiseKind::Depolarize1
                                                                                     : NoiseKind::Depolarize2;
      pl.noise.p1 = float_arg(0);
      pl.qs = qubits();
    } else if (name == "PAULI_CHANNEL_1") {
      pl.kind = 4;
      pl.noise.kind = NoiseKind::PauliChannel1;
      double v[3];
      for (int i = 0; i < 3; ++i)
        if (size_t(i) >= args.size() || !parse_f64(args[i], v[i]))
          throw err(ln, "PAULI_CHANNEL_1 needs three probabilities");
      pl.noise.p1 = v[0], pl.noise.p2 = v[1], pl.noise.p3 = v[2];
      pl.qs = qubits();
    } else if (name == "TICK") {
      pl.kind = 7;
    } else {
      throw err(ln, "unknown instruction '" + name + "'");
    }
    if (pl.kind == 2) {
      for (auto& s : pl.mpp) max_q = std::max(max_q, WidePauli::parse_with(s, std::nullopt).n);
    } else {
      for (size_t q : pl.qs) max_q = std::max(max_q, q + 1);
    }
    parsed.push_back(pl);
  }
  size_t n = declared ? *declared : max_q;
  if (n < max_q) throw SimError(ErrKind::Parse, "QUBITS " + std::to_string(n) + " but qubit " + std::to_string(max_q - 1) + " is used");
  Circuit c(n);
  for (auto& p : parsed) {
    try {
      switch (p.kind) {
        case 0: {
          size_t k = p.g.arity();
          if (p.g.g == G::Diagonal || p.g.g == G::Monomial) {
            c.gate(p.g, p.qs);
            break;
          }
          if (k == 0 || p.qs.size() % k != 0)
            throw err(p.ln, p.g.name() + " takes groups of " + std::to_string(k) + " qubits");
          for (size_t i = 0; i < p.qs.size(); i += k)
            c.gate(p.g, std::vector<size_t>(p.qs.begin() + i, p.qs.begin() + i + k));
          break;
        }
        case 1:
          for (size_t q : p.qs) {
            Op o;
            o.kind = OpKind::Measure;
            if (q >= n) throw SimError(ErrKind::QubitOutOfRange, "qubit out of range");
            o.pauli = n <= 64 ? Pauli::single(n, q, p.pk) : Pauli::identity(n);
            o.wide.n = n;
            o.wide.sites = {{q, uint8_t(p.pk == PauliKind::X ? 1 : p.pk == PauliKind::Z ? 2 : 3)}};
            c.push(o);
          }
          break;
        case 2:
          for (auto& s : p.mpp) {
            Op o;
            o.kind = OpKind::Measure;
            o.wide = WidePauli::parse_with(s, n);
            o.pauli = n <= 64 ? Pauli::from_string(n, s) : Pauli::identity(n);
            c.push(o);
          }
          break;
        case 3:
          for (size_t q : p.qs) {
            Op o;
            o.kind = OpKind::Reset;
            o.qubit = q;
            c.push(o);
          }
          break;
        case 4: {
          size_t k = p.noise.arity();
          if (p.qs.size() % k != 0) throw err(p.ln, "noise takes groups of " + std::to_string(k) + " qubits");
          for (size_t i = 0; i < p.qs.size(); i += k) {
            Op o;
            o.kind = OpKind::NoiseOp;
            o.noise = p.noise;
            o.qubits = std::vector<size_t>(p.qs.begin() + i, p.qs.begin() + i + k);
            c.push(o);
          }
          break;
        }
        case 5: case 6: {
          size_t m = c.num_measurements();
          for (size_t k : p.recs)
            if (k == 0 || k > m) throw SimError(ErrKind::Invalid, "rec[-" + std::to_string(k) + "] out of range");
          Op o;
          o.kind = p.kind == 5 ? OpKind::Detector : OpKind::Observable;
          o.lookback = p.recs;
          o.index = p.index;
          c.ops.push_back(o);
          break;
        }
        case 7: {
          Op o;
          o.kind = OpKind::Tick;
          c.ops.push_back(o);
          break;
        }
      }
    } catch (SimError& e) {
      if (e.kind == ErrKind::Parse) throw;
      throw err(p.ln, e.what());
    }
  }
  return c;
}

// ---------------------------------------------------------------------------
// StateVector<C64>: src/state/vector.rs
// ---------------------------------------------------------------------------
constexpr size_t BLOCK = size_t(1) << 12;  // vector.rs:192

// Bits of `v` deposited at the zero positions of `mask` (ascending order).
inline uint64_t deposit_skip(uint64_t v, uint64_t mask) {
  uint64_t out = 0;
  int vb = 0;
  for (int b = 0; b < 64 && (v >> vb); ++b) {
    if ((mask >> b) & 1) continue;
    out |= ((v >> vb) & 1ull) << b;
    ++vb;
  }
  return out;
}
// Faster insertion of zero bits at the (few) sorted positions in `pos`.
inline uint64_t insert_zeros(uint64_t v, const std::vector<int>& pos_sorted) {
  for (int b : pos_sorted) v = ((v >> b) << (b + 1)) | (v & ((1ull << b) - 1));
  return v;
}

struct StateVector {
  size_t n = 0;
  std::vector<C64> amp;

  static constexpr size_t MAX_QUBITS = 32;  // the reference asserts 30 (vector.rs:30)
  static StateVector basis_state(size_t n, uint64_t x) {  // vector.rs:29-34
    if (n > MAX_QUBITS) throw SimError(ErrKind::Invalid, "state vector of too many qubits");
    StateVector s;
    s.n = n;
    s.amp.assign(size_t(1) << n, C64());
    s.amp[x & mask_n(n)] = C64(1.0, 0.0);
    return s;
  }
  static StateVector zero_state(size_t n) { return basis_state(n, 0); }
  static StateVector plus_state(size_t n) {  // vector.rs:36-42
    StateVector s;
    s.n = n;
    s.amp.assign(size_t(1) << n, sqrt2_pow(-int64_t(n)));
    return s;
  }
  static StateVector from_amplitudes(size_t n, std::vector<C64> a) {
    if (a.size() != (size_t(1) << n)) throw SimError(ErrKind::Invalid, "amplitudes for n qubits");
    StateVector s;
    s.n = n;
    s.amp = std::move(a);
    return s;
  }

  // for_each_fiber (vector.rs:191-301): every fiber of 2^k amplitudes agreeing
  // off the gate qubits, in local little-endian order; fibers are independent,
  // so the traversal (blocks of 4096, high qubits splitting the vector) only
  // sets locality.  Here: fibers enumerated by their compressed base, in
  // contiguous chunks per thread.
  template <class F>
  void for_each_fiber(const std::vector<size_t>& qubits, const F& f) {
    size_t k = qubits.size();
    size_t gd = size_t(1) << k;
    std::vector<int> pos;
    uint64_t gmask = 0;
    for (size_t q : qubits) pos.push_back(int(q)), gmask |= 1ull << q;
    std::sort(pos.begin(), pos.end());
    std::vector<uint64_t> off(gd);
    for (size_t b = 0; b < gd; ++b) {
      uint64_t o = 0;
      for (size_t j = 0; j < k; ++j)
        if ((b >> j) & 1) o |= 1ull << qubits[j];
      off[b] = o;
    }
    int64_t nfib = int64_t(amp.size() >> k);
    C64* a = amp.data();
#pragma omp parallel
    {
      std::vector<C64> v(gd), w(gd);
#pragma omp for schedule(static)
      for (int64_t fi = 0; fi < nfib; ++fi) {
        uint64_t base = insert_zeros(uint64_t(fi), pos);
        for (size_t b = 0; b < gd; ++b) v[b] = a[base | off[b]];
        f(base, v.data(), w.data());
        for (size_t b = 0; b < gd; ++b) a[base | off[b]] = v[b];
      }
    }
  }

  // vector.rs:67-93
  void apply_matrix(const std::vector<C64>& m, const std::vector<size_t>& qubits) {
    check_qubits(qubits, n);
    size_t k = qubits.size(), gd = size_t(1) << k;
    if (m.size() != gd * gd) throw SimError(ErrKind::Invalid, "matrix size");
    std::vector<std::vector<std::pair<size_t, C64>>> nz(gd);
    for (size_t a = 0; a < gd; ++a)
      for (size_t b = 0; b < gd; ++b)
        if (!is_exactly_zero(m[a * gd + b])) nz[a].push_back({b, m[a * gd + b]});
    for_each_fiber(qubits, [&](uint64_t, C64* v, C64* w) {
      for (size_t a = 0; a < gd; ++a) {
        C64 acc;
        for (auto& bc : nz[a])
          if (!is_exactly_zero(v[bc.first])) acc = cadd(acc, cmul(bc.second, v[bc.first]));
        w[a] = acc;
      }
      for (size_t a = 0; a < gd; ++a) v[a] = w[a];
    });
  }

  // vector.rs:96-139
  void apply_monomial(const MonomialGate& g, const std::vector<size_t>& qubits) {
    check_qubits(qubits, n);
    size_t k = qubits.size();
    if (k != g.k) throw SimError(ErrKind::Arity, "monomial arity");
    bool affine_identity = g.shift == 0;
    for (size_t i = 0; i < k; ++i) affine_identity &= g.rows[i] == (1ull << i);
    if (affine_identity && k > 16) {
      // A diagonal over many qubits (e.g. the whole register): the reference's
      // 2^k image table does not fit, so each amplitude evaluates its own
      // image (the same phasor -> C64 conversion and the same "phase != 1"
      // and "amplitude != 0" skips as the table path).
      int64_t N = int64_t(amp.size());
      C64* a = amp.data();
      const C64 one(1.0, 0.0);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < N; ++i) {
        if (is_exactly_zero(a[i])) continue;
        uint64_t x = 0;
        for (size_t j = 0; j < k; ++j) x |= ((uint64_t(i) >> qubits[j]) & 1ull) << j;
        C64 c = from_phasor(g.apply_to_basis(x).first);
        if (!ceq(c, one)) a[i] = cmul(c, a[i]);
      }
      return;
    }
    size_t gd = size_t(1) << k;
    std::vector<std::pair<C64, size_t>> images(gd);
    for (size_t x = 0; x < gd; ++x) {
      auto [s, y] = g.apply_to_basis(x);
      images[x] = {from_phasor(s), size_t(y)};
    }
    bool diagonal = true;
    for (size_t x = 0; x < gd; ++x) diagonal &= images[x].second == x;
    const C64 one(1.0, 0.0);
    std::vector<std::pair<size_t, C64>> phased;
    std::vector<char> unit(gd);
    for (size_t x = 0; x < gd; ++x) {
      unit[x] = ceq(images[x].first, one);
      if (!unit[x]) phased.push_back({x, images[x].first});
    }
    if (diagonal) {
      if (phased.empty()) return;  // no amplitude changes
      for_each_fiber(qubits, [&](uint64_t, C64* v, C64*) {
        for (auto& xc : phased)
          if (!is_exactly_zero(v[xc.first])) v[xc.first] = cmul(xc.second, v[xc.first]);
      });
    } else {
      for_each_fiber(qubits, [&](uint64_t, C64* v, C64* w) {
        for (size_t x = 0; x < gd; ++x) w[images[x].second] = unit[x] ? v[x] : cmul(images[x].first, v[x]);
        for (size_t x = 0; x < gd; ++x) v[x] = w[x];
      });
    }
  }

  // for_each_pair (vector.rs:307-331): pairs {c, c^x}, c with the top bit of x clear.
  template <class F>
  void for_each_pair(uint64_t x, const F& f) {
    int h = 63 - __builtin_clzll(x);
    std::vector<int> pos{h};
    int64_t npairs = int64_t(amp.size() >> 1);
    C64* a = amp.data();
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < npairs; ++p) {
      uint64_t c = insert_zeros(uint64_t(p), pos);
      f(c, a[c], a[c ^ x]);
    }
  }

  // vector.rs:143-164
  void apply_pauli(const Pauli& p) {
    if (p.n != n) throw SimError(ErrKind::Invalid, "apply_pauli: register size");
    uint64_t xm = p.x, zm = p.z;
    uint8_t ph = p.phase;
    C64 ip[4] = {i_pow(0), i_pow(1), i_pow(2), i_pow(3)};
    auto k_of = [=](uint64_t c) { return (ph + 2 * popc(zm & c)) & 3; };
    if (xm == 0) {
      int64_t N = int64_t(amp.size());
      C64* a = amp.data();
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < N; ++c) {
        int k = k_of(uint64_t(c));
        if (k != 0 && !is_exactly_zero(a[c])) a[c] = cmul(ip[k], a[c]);
      }
    } else {
      for_each_pair(xm, [&](uint64_t c, C64& a, C64& b) {
        C64 na = cmul(ip[k_of(c ^ xm)], b);
        C64 nb = cmul(ip[k_of(c)], a);
        a = na;
        b = nb;
      });
    }
  }

  // vector.rs:168-188
  StateVector kron(const StateVector& o) const {
    size_t nn = n + o.n;
    if (nn > MAX_QUBITS) throw SimError(ErrKind::Invalid, "state vector of too many qubits");
    StateVector s;
    s.n = nn;
    s.amp.assign(size_t(1) << nn, C64());
    size_t la = amp.size();
    int64_t lb = int64_t(o.amp.size());
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < lb; ++j) {
      C64 b = o.amp[j];
      if (is_exactly_zero(b)) continue;
      for (size_t i = 0; i < la; ++i)
        if (!is_exactly_zero(amp[i])) s.amp[size_t(j) * la + i] = cmul(amp[i], b);
    }
    return s;
  }

  // par_sum (vector.rs:334-350): the pairwise order, forked at 2^14.
  template <class F>
  static C64 par_sum_rec(size_t lo, size_t hi, const F& f) {
    size_t len = hi - lo;
    if (len <= 8) {
      C64 acc;
      for (size_t i = lo; i < hi; ++i) acc = cadd(acc, f(i));
      return acc;
    }
    size_t mid = lo + len / 2;
    C64 a, b;
    if (len >= (size_t(1) << 22)) {
#pragma omp task shared(a)
      a = par_sum_rec(lo, mid, f);
#pragma omp task shared(b)
      b = par_sum_rec(mid, hi, f);
#pragma omp taskwait
    } else {
      a = par_sum_rec(lo, mid, f);
      b = par_sum_rec(mid, hi, f);
    }
    return cadd(a, b);
  }
  template <class F>
  static C64 par_sum(size_t lo, size_t hi, const F& f) {
    C64 r;
#pragma omp parallel
#pragma omp single
    r = par_sum_rec(lo, hi, f);
    return r;
  }

  // vector.rs:397-406
  C64 norm_sq() const {
    const C64* a = amp.data();
    return par_sum(0, amp.size(), [a](size_t i) { return is_exactly_zero(a[i]) ? C64() : abs_sq(a[i]); });
  }
  C64 amplitude(uint64_t x) const { return amp[x & mask_n(n)]; }
  // vector.rs:412-429
  C64 expectation(const Pauli& p) const {
    if (p.n != n) throw SimError(ErrKind::Invalid, "expectation: operator on the wrong register");
    uint64_t xm = p.x, zm = p.z;
    uint8_t ph = p.phase;
    const C64* a = amp.data();
    return par_sum(0, amp.size(), [=](size_t c) {
      if (is_exactly_zero(a[c]) || is_exactly_zero(a[c ^ xm])) return C64();
      int k = (ph + 2 * popc(zm & c)) & 3;
      return cmul(cconj(a[c ^ xm]), cmul(i_pow(k), a[c]));
    });
  }
  // vector.rs:431-443
  C64 inner(const StateVector& o) const {
    if (o.n != n) throw SimError(ErrKind::Invalid, "inner: register sizes differ");
    const C64* a = amp.data();
    const C64* b = o.amp.data();
    return par_sum(0, amp.size(), [=](size_t i) {
      if (is_exactly_zero(a[i]) || is_exactly_zero(b[i])) return C64();
      return cmul(cconj(a[i]), b[i]);
    });
  }
  // vector.rs:445-479
  C64 project(const Pauli& p, bool outcome) {
    if (!p.is_hermitian()) throw SimError(ErrKind::Invalid, "projector of non-Hermitian Pauli");
    uint64_t xm = p.x, zm = p.z;
    uint8_t ph = p.phase;
    C64 one(1.0, 0.0);
    C64 half(0.5, 0.0);  // (1 + 1)^{-1}
    C64 sgn[4];
    for (int k = 0; k < 4; ++k) sgn[k] = outcome ? cneg(i_pow(k)) : i_pow(k);
    auto k_of = [=](uint64_t c) { return (ph + 2 * popc(zm & c)) & 3; };
    (void)one;
    if (xm == 0) {
      int64_t N = int64_t(amp.size());
      C64* a = amp.data();
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < N; ++c)
        if (!is_exactly_zero(a[c])) a[c] = cmul(cadd(a[c], cmul(sgn[k_of(uint64_t(c))], a[c])), half);
    } else {
      for_each_pair(xm, [&](uint64_t c, C64& a, C64& b) {
        uint64_t d = c ^ xm;
        C64 na = cmul(cadd(a, cmul(sgn[k_of(d)], b)), half);
        C64 nb = cmul(cadd(b, cmul(sgn[k_of(c)], a)), half);
        a = na;
        b = nb;
      });
    }
    return norm_sq();
  }
  // vector.rs:481-488
  void scale(C64 c) {
    int64_t N = int64_t(amp.size());
    C64* a = amp.data();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i)
      if (!is_exactly_zero(a[i])) a[i] = cmul(a[i], c);
  }

  // vector.rs:364-395
  void apply_gate(const Gate& gate, const std::vector<size_t>& qubits) {
    check_qubits(qubits, n);
    if (qubits.size() != gate.arity())
      throw SimError(ErrKind::Arity, "gate " + gate.name() + " acts on " + std::to_string(gate.arity()) +
                                         " qubits, " + std::to_string(qubits.size()) + " given");
    if (gate.g == G::PauliG) {
      apply_pauli(gate.pauli.embed(n, qubits));
      return;
    }
    if (auto m = gate.monomial()) {
      apply_monomial(*m, qubits);
      return;
    }
    if (auto m = gate.matrix()) {
      apply_matrix(*m, qubits);
      return;
    }
    throw SimError(ErrKind::NotRepresentable, "gate " + gate.name() + " in the scalar type");
  }

  // vector.rs:494-540: one-pass sampling; returns basis indices
  std::vector<uint64_t> sample_from_uniforms(const std::vector<double>& draws) const {
    const C64* a = amp.data();
    size_t len = amp.size();
    size_t bl = std::min(BLOCK, len);
    size_t nb = (len + bl - 1) / bl;
    std::vector<double> weights(nb);
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < int64_t(nb); ++b) {
      double s = 0.0;
      size_t e = std::min(len, size_t(b + 1) * bl);
      for (size_t i = size_t(b) * bl; i < e; ++i) s += norm_sqr(a[i]);
      weights[b] = s;
    }
    double total = 0.0;
    for (double w : weights) total += w;
    if (total <= 0.0) throw SimError(ErrKind::ZeroState, "state vanished: sample");
    size_t shots = draws.size();
    std::vector<std::pair<double, size_t>> us(shots);
    for (size_t k = 0; k < shots; ++k) us[k] = {draws[k] * total, k};
    std::sort(us.begin(), us.end(), [](const auto& x, const auto& y) {
      if (x.first != y.first) return x.first < y.first;
      return false;
    });
    std::vector<uint64_t> out(shots);
    size_t next = 0;
    double acc = 0.0;
    for (size_t b = 0; b < nb; ++b) {
      if (next == shots) break;
      double hi = acc + weights[b];
      bool last_block = b + 1 == nb;
      if (us[next].first < hi || last_block) {
        double run = acc;
        size_t start = b * bl, end = std::min(start + bl, len);
        size_t idx = start;
        while (next < shots && (us[next].first < hi || last_block)) {
          double u = us[next].first;
          while (idx + 1 < end && run + norm_sqr(a[idx]) <= u) {
            run += norm_sqr(a[idx]);
            idx += 1;
          }
          size_t pick = idx;
          while (is_exactly_zero(a[pick]) && pick > start) pick -= 1;
          out[us[next].second] = pick;
          next += 1;
        }
      }
      acc = hi;
    }
    return out;
  }
  std::vector<uint64_t> sample(StdRng& rng, size_t shots) const {
    std::vector<double> d(shots);
    // the uniforms are drawn first, in shot order (vector.rs:505)
    for (size_t k = 0; k < shots; ++k) d[k] = rng.gen_f64();
    return sample_from_uniforms(d);
  }

  // ---- provided trait methods: src/state/mod.rs:93-234 ----
  double probability(uint64_t x) const { return norm_sqr(amplitude(x)) / norm_sq().re; }
  bool measure(const Pauli& p, StdRng& rng) {  // mod.rs:113-131
    if (!p.is_hermitian()) throw SimError(ErrKind::Invalid, "measured operator is not Hermitian");
    double e = expectation(p).re;
    double nn = norm_sq().re;
    double p_plus = (1.0 + e / nn) / 2.0;
    if (!std::isnan(p_plus)) p_plus = std::min(1.0, std::max(0.0, p_plus));
    bool outcome;
    if (p_plus > 1.0 - 1e-12) outcome = false;
    else if (p_plus < 1e-12) outcome = true;
    else outcome = rng.gen_f64() >= p_plus;
    project(p, outcome);
    return outcome;
  }
  // mod.rs:134-165; returns -1 for no outcome
  int apply_op(const Op& op, StdRng& rng) {
    switch (op.kind) {
      case OpKind::GateOp: apply_gate(op.gate, op.qubits); return -1;
      case OpKind::Measure: return measure(op.pauli, rng) ? 1 : 0;
      case OpKind::Reset: {
        if (measure(Pauli::zq(n, op.qubit), rng)) apply_gate(Gate::named(G::X), {op.qubit});
        return -1;
      }
      case OpKind::NoiseOp: {
        auto e = op.noise.sample(rng);
        if (e) {
          Pauli p = Pauli::identity(n);
          for (size_t j = 0; j < op.qubits.size(); ++j)
            p.set_raw_bits(op.qubits[j], (e->first >> j) & 1, (e->second >> j) & 1);
          Gate g;
          g.g = G::PauliG;
          g.pauli = p.restrict_to(op.qubits);
          apply_gate(g, op.qubits);
        }
        return -1;
      }
      default: return -1;
    }
  }
  // mod.rs:168-183
  std::vector<uint8_t> run(const Circuit& c, StdRng& rng) {
    if (c.n != n) throw SimError(ErrKind::Invalid, "circuit on a different register");
    std::vector<uint8_t> rec;
    for (auto& op : c.ops) {
      int r = apply_op(op, rng);
      if (r >= 0) rec.push_back(uint8_t(r));
    }
    return rec;
  }
  // mod.rs:220-233
  void normalize() {
    double nn = norm_sq().re;
    if (nn <= 0.0) throw SimError(ErrKind::ZeroState, "state vanished: normalize");
    double l = -std::log2(nn);
    C64 c = std::fabs(l - std::round(l)) < 1e-9 ? sqrt2_pow(int64_t(std::round(l))) : C64(1.0 / std::sqrt(nn), 0.0);
    scale(c);
  }
  // mod.rs:93-101
  C64 expectation_sum(const std::vector<std::pair<Pauli, C64>>& h) const {
    std::vector<C64> terms(h.size());
    for (size_t i = 0; i < h.size(); ++i) terms[i] = cmul(h[i].second, expectation(h[i].first));
    return pairwise_sum(terms.data(), terms.size());
  }
};

// ---------------------------------------------------------------------------
// A sparse restatement of the same gate arithmetic (index -> amplitude, exact
// zeros dropped), for permutation/diagonal-heavy registers too large for a
// dense CPU vector: the views, image tables and skip rules are the dense
// ones above, applied to the stored entries only.
// ---------------------------------------------------------------------------
struct SparseState {
  size_t n = 0;
  std::vector<std::pair<uint64_t, C64>> ent;  // sorted by index

  static SparseState zero_state(size_t n) {
    SparseState s;
    s.n = n;
    s.ent.push_back({0, C64(1.0, 0.0)});
    return s;
  }
  void canonical() {
    std::sort(ent.begin(), ent.end(), [](auto& a, auto& b) { return a.first < b.first; });
    std::vector<std::pair<uint64_t, C64>> out;
    for (auto& e : ent)
      if (!is_exactly_zero(e.second)) out.push_back(e);
    ent.swap(out);
  }
  static uint64_t local_of(uint64_t idx, const std::vector<size_t>& qs) {
    uint64_t x = 0;
    for (size_t j = 0; j < qs.size(); ++j) x |= ((idx >> qs[j]) & 1ull) << j;
    return x;
  }
  static uint64_t with_local(uint64_t idx, const std::vector<size_t>& qs, uint64_t y) {
    for (size_t j = 0; j < qs.size(); ++j) idx = (idx & ~(1ull << qs[j])) | (((y >> j) & 1ull) << qs[j]);
    return idx;
  }
  void apply_monomial(const MonomialGate& g, const std::vector<size_t>& qs) {
    const C64 one(1.0, 0.0);
    int64_t m = int64_t(ent.size());
    // the same per-image conversion as the dense table path
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
      auto& e = ent[i];
      uint64_t x = local_of(e.first, qs);
      auto [s, y] = g.apply_to_basis(x);
      C64 c = from_phasor(s);
      if (!ceq(c, one)) e.second = cmul(c, e.second);
      e.first = with_local(e.first, qs, y);
    }
    canonical();
  }
  void apply_matrix(const std::vector<C64>& mat, const std::vector<size_t>& qs) {
    size_t k = qs.size(), gd = size_t(1) << k;
    uint64_t gmask = 0;
    for (size_t q : qs) gmask |= 1ull << q;
    std::sort(ent.begin(), ent.end(), [&](auto& a, auto& b) {
      uint64_t ba = a.first & ~gmask, bb = b.first & ~gmask;
      return ba != bb ? ba < bb : a.first < b.first;
    });
    std::vector<std::pair<uint64_t, C64>> out;
    size_t i = 0;
    std::vector<C64> v(gd), w(gd);
    while (i < ent.size()) {
      uint64_t base = ent[i].first & ~gmask;
      std::fill(v.begin(), v.end(), C64());
      while (i < ent.size() && (ent[i].first & ~gmask) == base) {
        v[local_of(ent[i].first, qs)] = ent[i].second;
        ++i;
      }
      for (size_t a = 0; a < gd; ++a) {
        C64 acc;
        for (size_t b = 0; b < gd; ++b) {
          C64 mc = mat[a * gd + b];
          if (!is_exactly_zero(mc) && !is_exactly_zero(v[b])) acc = cadd(acc, cmul(mc, v[b]));
        }
        w[a] = acc;
      }
      for (size_t a = 0; a < gd; ++a) out.push_back({with_local(base, qs, a), w[a]});
    }
    ent.swap(out);
    canonical();
  }
  void apply_gate(const Gate& gate, const std::vector<size_t>& qubits) {
    check_qubits(qubits, n);
    if (qubits.size() != gate.arity()) throw SimError(ErrKind::Arity, "arity");
    if (gate.g == G::PauliG) throw SimError(ErrKind::Unsupported, "sparse oracle: Pauli gates");
    if (auto m = gate.monomial()) return apply_monomial(*m, qubits);
    if (auto m = gate.matrix()) return apply_matrix(*m, qubits);
    throw SimError(ErrKind::NotRepresentable, "gate");
  }
};

}  // namespace ref
