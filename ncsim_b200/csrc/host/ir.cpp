// Parsing, printing and lowering of the host-side circuit IR.
#include "ir.hpp"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <sstream>

namespace ncsim {

namespace {

std::string upcase(std::string s) {
  for (char& c : s) c = char(std::toupper((unsigned char)c));
  return s;
}

std::string strip(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

std::vector<std::string> split_on(const std::string& s, char sep) {
  std::vector<std::string> v(1);
  for (char c : s) {
    if (c == sep) v.emplace_back();
    else v.back().push_back(c);
  }
  return v;
}

bool to_u64(const std::string& s0, uint64_t& v) {
  std::string s = strip(s0);
  if (s.empty() || !std::isdigit((unsigned char)s[0])) return false;
  errno = 0;
  char* e = nullptr;
  unsigned long long r = std::strtoull(s.c_str(), &e, 10);
  if (errno || *e) return false;
  v = r;
  return true;
}

bool to_i64(const std::string& s0, int64_t& v) {
  std::string s = strip(s0);
  if (s.empty()) return false;
  errno = 0;
  char* e = nullptr;
  long long r = std::strtoll(s.c_str(), &e, 10);
  if (errno || *e) return false;
  v = r;
  return true;
}

bool to_f64(const std::string& s0, double& v) {
  std::string s = strip(s0);
  if (s.empty()) return false;
  char* e = nullptr;
  v = std::strtod(s.c_str(), &e);
  return *e == 0;
}

Error parse_error(const std::string& m) { return Error(NCSIM_ERR_PARSE, m); }

uint64_t mask_bits(uint32_t n) { return n >= 64 ? ~uint64_t(0) : ((uint64_t(1) << n) - 1); }

// letter on qubit q of a Pauli, keeping the letter phase (pauli/mod.rs:195-206)
void set_letter(PauliOp& p, uint32_t q, char letter) {
  const uint64_t b = uint64_t(1) << q;
  if ((p.x & b) && (p.z & b)) p.phase = (p.phase + 3) & 3;
  p.x &= ~b;
  p.z &= ~b;
  if (letter == 'X' || letter == 'Y') p.x |= b;
  if (letter == 'Z' || letter == 'Y') p.z |= b;
  if (letter == 'Y') p.phase = (p.phase + 1) & 3;
}

}  // namespace

std::string fmt_f64(double v) {
  char b[40];
  std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}

// ---------------------------------------------------------------------------
PauliSites parse_pauli_sites(const std::string& text, int64_t nreg) {
  auto bad = [&](const std::string& m) { return parse_error("Pauli '" + text + "': " + m); };
  std::string rest = strip(text);
  uint32_t ph = 0;
  static const std::pair<const char*, uint32_t> prefixes[] = {{"-i", 3}, {"+i", 1}, {"-", 2}, {"+", 0}, {"i", 1}};
  for (auto& pr : prefixes) {
    size_t L = std::strlen(pr.first);
    if (rest.compare(0, L, pr.first) == 0) {
      rest = strip(rest.substr(L));
      if (!rest.empty() && rest[0] == '*') rest = strip(rest.substr(1));
      ph = pr.second;
      break;
    }
  }
  auto bits_of = [](char c) -> uint8_t { return c == 'X' ? 1 : c == 'Z' ? 2 : c == 'Y' ? 3 : 0; };
  PauliSites p;
  p.phase = ph;
  const bool dense = !rest.empty() && rest.find_first_not_of("IXYZ_") == std::string::npos;
  if (dense) {
    if (rest.size() > MAX_CIRCUIT_QUBITS) throw bad("more than " + std::to_string(MAX_CIRCUIT_QUBITS) + " qubits");
    if (nreg >= 0 && size_t(nreg) != rest.size())
      throw bad(std::to_string(rest.size()) + " letters for " + std::to_string(nreg) + " qubits");
    p.n = uint32_t(rest.size());
    for (uint32_t q = 0; q < p.n; ++q)
      if (uint8_t b = bits_of(rest[q])) p.sites.push_back({q, b});
    return p;
  }
  std::string tok;
  auto flush = [&] {
    if (tok.empty()) return;
    std::string t;
    t.swap(tok);
    if (t == "1") return;
    char c = t[0];
    if (c == '_') c = 'I';
    if (c != 'I' && c != 'X' && c != 'Y' && c != 'Z') throw bad("token '" + t + "'");
    uint64_t q;
    if (!to_u64(t.substr(1), q) || t.size() < 2) throw bad("token '" + t + "'");
    if (q >= MAX_CIRCUIT_QUBITS) throw bad("qubit " + std::to_string(q) + " above the register limit");
    for (auto& s : p.sites)
      if (s.first == q) throw bad("qubit " + std::to_string(q) + " repeated");
    p.sites.push_back({uint32_t(q), bits_of(c)});  // identity letters hold a place until the sort
  };
  for (char c : rest) {
    if (c == '*' || std::isspace((unsigned char)c)) flush();
    else tok.push_back(c);
  }
  flush();
  uint64_t n = 0;
  if (nreg >= 0) n = uint64_t(nreg);
  else
    for (auto& s : p.sites) n = std::max<uint64_t>(n, uint64_t(s.first) + 1);
  p.n = uint32_t(n);
  for (auto& s : p.sites)
    if (s.first >= n) throw bad("qubit " + std::to_string(s.first) + " out of range for " + std::to_string(n) + " qubits");
  p.sites.erase(std::remove_if(p.sites.begin(), p.sites.end(), [](const std::pair<uint32_t, uint8_t>& s) { return s.second == 0; }),
                p.sites.end());
  std::sort(p.sites.begin(), p.sites.end());
  return p;
}

PauliOp pauli_from_sites(const PauliSites& s) {
  if (s.n > 64) throw parse_error("Paulis on more than 64 qubits have no one-word form");
  PauliOp p;
  p.n = s.n;
  uint32_t ys = 0;
  for (auto& st : s.sites) {
    if (st.second & 1) p.x |= uint64_t(1) << st.first;
    if (st.second & 2) p.z |= uint64_t(1) << st.first;
    ys += st.second == 3;
  }
  p.phase = (s.phase + ys) & 3;
  return p;
}

PauliOp parse_pauli(const std::string& text, int64_t nreg) {
  PauliSites s = parse_pauli_sites(text, nreg);
  if (s.n > 64) throw parse_error("Pauli '" + text + "': more than 64 qubits");
  return pauli_from_sites(s);
}

static std::string pauli_sparse(const PauliOp& p) {
  const uint32_t ys = uint32_t(__builtin_popcountll(p.x & p.z));
  const uint32_t k = (p.phase + 4 - (ys & 3)) & 3;  // the letter phase
  static const char* pre[] = {"", "i*", "-", "-i*"};
  std::string body;
  for (uint32_t q = 0; q < p.n; ++q) {
    bool bx = (p.x >> q) & 1, bz = (p.z >> q) & 1;
    if (!bx && !bz) continue;
    if (!body.empty()) body += "*";
    body += (bx && bz) ? 'Y' : bx ? 'X' : 'Z';
    body += std::to_string(q);
  }
  if (body.empty()) {
    static const char* sc[] = {"1", "i", "-1", "-i"};
    return sc[k];
  }
  return pre[k] + body;
}

// ---------------------------------------------------------------------------
uint64_t PhasePolyIR::eval(uint64_t x) const {
  const uint64_t mm = mask_bits(bits);
  uint64_t f = constant;
  for (size_t t = 0; t < coeffs.size(); ++t) {
    bool all = true;
    for (uint64_t l : parities[t])
      if (!(__builtin_popcountll(l & mask_bits(nvars) & x) & 1)) {
        all = false;
        break;
      }
    if (all) f += coeffs[t];
  }
  return f & mm;
}

bool MonomialIR::affine_identity() const {
  if (shift) return false;
  for (uint32_t i = 0; i < k; ++i)
    if (rows[i] != (uint64_t(1) << i)) return false;
  return true;
}

static size_t gf2_rank_of(std::vector<uint64_t> r) {
  size_t rank = 0;
  for (int bit = 0; bit < 64 && rank < r.size(); ++bit) {
    size_t p = rank;
    while (p < r.size() && !((r[p] >> bit) & 1)) ++p;
    if (p == r.size()) continue;
    std::swap(r[p], r[rank]);
    for (size_t i = 0; i < r.size(); ++i)
      if (i != rank && ((r[i] >> bit) & 1)) r[i] ^= r[rank];
    ++rank;
  }
  return rank;
}

uint32_t GateIR::arity() const {
  switch (kind) {
    case GateKind::Cx: case GateKind::Cy: case GateKind::Cz: case GateKind::Swap: case GateKind::Cs:
    case GateKind::Csdg: case GateKind::CPhase:
      return 2;
    case GateKind::Ccz: case GateKind::Ccx: return 3;
    case GateKind::Diagonal: return poly.nvars;
    case GateKind::Monomial: return mono.k;
    case GateKind::Pauli: return pauli.n;
    case GateKind::Unitary: return uk;
    default: return 1;
  }
}

static std::string poly_text(const PhasePolyIR& p) {
  std::string s = std::to_string(p.bits) + ";" + std::to_string(p.constant);
  for (size_t t = 0; t < p.coeffs.size(); ++t) {
    s += ";" + std::to_string(p.coeffs[t]) + ":";
    for (size_t i = 0; i < p.parities[t].size(); ++i) s += (i ? "," : "") + std::to_string(p.parities[t][i]);
  }
  return s;
}

std::string GateIR::text() const {
  static const char* names[] = {"I", "X", "Y", "Z", "H", "S", "S_DAG", "SQRT_X", "SQRT_X_DAG", "SQRT_Y", "SQRT_Y_DAG",
                                "T", "T_DAG", "CX", "CY", "CZ", "SWAP", "CS", "CS_DAG", "CCZ", "CCX"};
  switch (kind) {
    case GateKind::Phase: return "PHASE(" + std::to_string(pk) + "," + std::to_string(pbits) + ")";
    case GateKind::CPhase: return "CPHASE(" + std::to_string(pk) + "," + std::to_string(pbits) + ")";
    case GateKind::Rx: return "RX(" + fmt_f64(theta) + ")";
    case GateKind::Ry: return "RY(" + fmt_f64(theta) + ")";
    case GateKind::Rz: return "RZ(" + fmt_f64(theta) + ")";
    case GateKind::Diagonal: return "DIAG(" + poly_text(poly) + ")";
    case GateKind::Monomial: {
      std::string s = "MONOMIAL(";
      for (uint32_t i = 0; i < mono.k; ++i) s += (i ? "," : "") + std::to_string(mono.rows[i]);
      s += ";" + std::to_string(mono.shift) + ";" + poly_text(mono.phase) + ";" + std::to_string(mono.scalar.s2) + "," +
           std::to_string(mono.scalar.phase) + "," + std::to_string(mono.scalar.bits) + ")";
      return s;
    }
    case GateKind::Pauli: return "PAULI[" + pauli_sparse(pauli) + "]";
    case GateKind::Unitary: return "UNITARY[" + std::to_string(uk) + " qubits]";
    default: return names[int(kind)];
  }
}

// ---------------------------------------------------------------------------
// views and lowering
// ---------------------------------------------------------------------------
namespace {

MonomialIR diag_mono(uint32_t k, uint32_t bits, std::initializer_list<std::pair<int64_t, uint64_t>> terms) {
  MonomialIR m;
  m.k = k;
  for (uint32_t i = 0; i < k; ++i) m.rows.push_back(uint64_t(1) << i);
  m.phase.nvars = k;
  m.phase.bits = bits;
  const uint64_t mm = mask_bits(bits);
  for (auto& t : terms) {
    // a monomial prod_{v in vars} x_v: one parity per variable
    std::vector<uint64_t> pars;
    for (uint32_t v = 0; v < k; ++v)
      if ((t.second >> v) & 1) pars.push_back(uint64_t(1) << v);
    m.phase.parities.push_back(pars);
    m.phase.coeffs.push_back(uint64_t(emod(t.first, int64_t(mm) + 1)));
  }
  return m;
}

}  // namespace

// Gate::monomial (gate.rs:519-564); false when the gate has no monomial view
bool monomial_view(const GateIR& g, MonomialIR& m) {
  switch (g.kind) {
    case GateKind::I: m = diag_mono(1, 1, {}); return true;
    case GateKind::X: m = diag_mono(1, 1, {}); m.shift = 1; return true;
    case GateKind::Y:  // MonomialGate::pauli(Y): shift 1, phase x0 mod 2, scalar i
      m = diag_mono(1, 1, {{1, 1}});
      m.shift = 1;
      m.scalar = Phase::make(0, 1, 2);
      return true;
    case GateKind::Z: m = diag_mono(1, 1, {{1, 1}}); return true;
    case GateKind::S: m = diag_mono(1, 2, {{1, 1}}); return true;
    case GateKind::Sdg: m = diag_mono(1, 2, {{3, 1}}); return true;
    case GateKind::T: m = diag_mono(1, 3, {{1, 1}}); return true;
    case GateKind::Tdg: m = diag_mono(1, 3, {{7, 1}}); return true;
    case GateKind::Phase: m = diag_mono(1, g.pbits, {{g.pk, 1}}); return true;
    case GateKind::CPhase: m = diag_mono(2, g.pbits, {{g.pk, 3}}); return true;
    case GateKind::Cz: m = diag_mono(2, 1, {{1, 3}}); return true;
    case GateKind::Cs: m = diag_mono(2, 2, {{1, 3}}); return true;
    case GateKind::Csdg: m = diag_mono(2, 2, {{3, 3}}); return true;
    case GateKind::Ccz: m = diag_mono(3, 1, {{1, 7}}); return true;
    case GateKind::Cx: m = diag_mono(2, 1, {}); m.rows = {1, 3}; return true;
    case GateKind::Cy: m = diag_mono(2, 2, {{1, 1}, {2, 3}}); m.rows = {1, 3}; return true;
    case GateKind::Swap: m = diag_mono(2, 1, {}); m.rows = {2, 1}; return true;
    case GateKind::Diagonal:
      m = MonomialIR();
      m.k = g.poly.nvars;
      for (uint32_t i = 0; i < m.k; ++i) m.rows.push_back(uint64_t(1) << i);
      m.phase = g.poly;
      return true;
    case GateKind::Monomial: m = g.mono; return true;
    default: return false;
  }
}

std::vector<CplxD> gate_matrix(const GateIR& g) {
  const double h = 0.5 * 1.41421356237309504880;  // sqrt2_pow(-1)
  switch (g.kind) {
    case GateKind::H: return {{h, 0}, {h, 0}, {h, 0}, {-h, 0}};
    case GateKind::SqrtX: return {{0.5, 0.5}, {0.5, -0.5}, {0.5, -0.5}, {0.5, 0.5}};
    case GateKind::SqrtXdg: return {{0.5, -0.5}, {0.5, 0.5}, {0.5, 0.5}, {0.5, -0.5}};
    case GateKind::SqrtY: return {{0.5, 0.5}, {-0.5, -0.5}, {0.5, 0.5}, {0.5, 0.5}};
    case GateKind::SqrtYdg: return {{0.5, -0.5}, {0.5, -0.5}, {-0.5, 0.5}, {0.5, -0.5}};
    case GateKind::Rx: {
      double c = std::cos(g.theta / 2.0), s = std::sin(g.theta / 2.0);
      return {{c, 0}, {0, -s}, {0, -s}, {c, 0}};
    }
    case GateKind::Ry: {
      double c = std::cos(g.theta / 2.0), s = std::sin(g.theta / 2.0);
      return {{c, 0}, {-s, 0}, {s, 0}, {c, 0}};
    }
    case GateKind::Rz:
      return {{std::cos(-g.theta / 2.0), std::sin(-g.theta / 2.0)}, {0, 0}, {0, 0},
              {std::cos(g.theta / 2.0), std::sin(g.theta / 2.0)}};
    case GateKind::Ccx: {
      std::vector<CplxD> m(64, CplxD{0, 0});
      for (int x = 0; x < 8; ++x) m[((x & 3) == 3 ? (x ^ 4) : x) * 8 + x] = {1, 0};
      return m;
    }
    case GateKind::Unitary: return g.umat;
    default: {
      MonomialIR mo;
      if (!monomial_view(g, mo)) throw Error(NCSIM_ERR_NOT_REPRESENTABLE, "gate " + g.text() + " has no matrix");
      const size_t d = size_t(1) << mo.k;
      std::vector<CplxD> m(d * d, CplxD{0, 0});
      for (uint64_t x = 0; x < d; ++x) {
        uint64_t y = mo.shift;
        for (uint32_t i = 0; i < mo.k; ++i)
          if (__builtin_popcountll(mo.rows[i] & x) & 1) y ^= uint64_t(1) << i;
        Cd v = mo.scalar.times(Phase::make(0, int64_t(mo.phase.eval(x)), mo.phase.bits)).value();
        m[y * d + x] = {v.re, v.im};
      }
      return m;
    }
  }
}

static PolyTerms poly_terms_for(const PhasePolyIR& p, const std::vector<uint32_t>& qubits, const Phase& scalar) {
  PolyTerms t;
  t.bits = p.bits;
  const uint64_t mm = mask_bits(p.bits);
  t.constant = p.constant & mm;
  t.term_start.push_back(0);
  for (size_t i = 0; i < p.coeffs.size(); ++i) {
    uint64_t c = p.coeffs[i] & mm;
    bool vanishes = false;
    std::vector<uint64_t> glob;
    for (uint64_t l : p.parities[i]) {
      uint64_t lm = l & mask_bits(p.nvars);
      if (!lm) vanishes = true;
      uint64_t gm = 0;
      for (uint32_t j = 0; j < p.nvars; ++j)
        if ((lm >> j) & 1) gm |= uint64_t(1) << qubits[j];
      glob.push_back(gm);
    }
    if (vanishes || !c) continue;
    if (glob.empty()) {
      t.constant = (t.constant + c) & mm;
      continue;
    }
    t.parities.insert(t.parities.end(), glob.begin(), glob.end());
    t.coeffs.push_back(c);
    t.term_start.push_back(uint32_t(t.parities.size()));
  }
  t.scalar_is_one = scalar.is_one();
  Cd sv = scalar.value();
  t.scalar = {sv.re, sv.im};
  if (p.bits <= 8) {
    t.root_table.resize(size_t(1) << p.bits);
    for (uint64_t f = 0; f < (uint64_t(1) << p.bits); ++f) {
      Cd v = scalar.times(Phase::make(0, int64_t(f), p.bits)).value();
      t.root_table[f] = {v.re, v.im};
    }
  }
  return t;
}

PolyTerms build_poly_terms(const PhasePolyIR& p, const std::vector<uint32_t>& qubits, const Phase& scalar) {
  return poly_terms_for(p, qubits, scalar);
}

LoweredOp lower_gate(const GateIR& g, const std::vector<uint32_t>& qubits, uint32_t n) {
  // check_qubits and the arity check of apply_gate (vector.rs:365-372)
  for (size_t i = 0; i < qubits.size(); ++i) {
    if (qubits[i] >= n) throw qubit_out_of_range(qubits[i], n);
    for (size_t j = 0; j < i; ++j)
      if (qubits[j] == qubits[i]) throw duplicate_qubit(qubits[i]);
  }
  if (qubits.size() != g.arity()) throw arity_error(g.text(), g.arity(), qubits.size());
  LoweredOp op;
  op.qubits = qubits;
  if (g.kind == GateKind::Pauli) {  // Pauli::embed (pauli/mod.rs:292-301)
    op.kind = LoweredKind::Pauli;
    for (size_t j = 0; j < qubits.size(); ++j) {
      op.x |= ((g.pauli.x >> j) & 1ull) << qubits[j];
      op.z |= ((g.pauli.z >> j) & 1ull) << qubits[j];
    }
    op.phase = g.pauli.phase & 3;
    return op;
  }
  if (g.kind == GateKind::Ccx) {
    // Its dense view (gate.rs:697-705) is a 0/1 permutation matrix, applied
    // exactly as a permutation table: the target flips when both controls
    // are set (not an affine map, so not a MonomialGate).
    op.kind = LoweredKind::Monomial;
    op.image.resize(8);
    op.matrix.assign(8, CplxD{1.0, 0.0});
    for (uint32_t x = 0; x < 8; ++x) op.image[x] = (x & 3) == 3 ? (x ^ 4) : x;
    return op;
  }
  MonomialIR mo;
  if (!monomial_view(g, mo)) {
    op.kind = LoweredKind::Dense;
    op.matrix = gate_matrix(g);
    if (qubits.size() > size_t(MAX_WIDE_DENSE_K))
      throw Error(NCSIM_ERR_UNSUPPORTED, "dense gates on more than " + std::to_string(MAX_WIDE_DENSE_K) + " qubits");
    return op;
  }
  if (mo.affine_identity() && mo.k > 10) {
    op.kind = LoweredKind::PhasePoly;
    op.poly = poly_terms_for(mo.phase, qubits, mo.scalar);
    return op;
  }
  if (mo.k > uint32_t(MAX_WIDE_MONOMIAL_K))
    throw Error(NCSIM_ERR_UNSUPPORTED, "monomial gates on more than " + std::to_string(MAX_WIDE_MONOMIAL_K) + " qubits");
  op.kind = LoweredKind::Monomial;
  const size_t d = size_t(1) << mo.k;
  op.image.resize(d);
  op.matrix.resize(d);
  for (uint64_t x = 0; x < d; ++x) {  // MonomialGate::apply_to_basis (gate.rs:157-169)
    uint64_t y = mo.shift;
    for (uint32_t i = 0; i < mo.k; ++i)
      if (__builtin_popcountll(mo.rows[i] & x) & 1) y ^= uint64_t(1) << i;
    Cd v = mo.scalar.times(Phase::make(0, int64_t(mo.phase.eval(x)), mo.phase.bits)).value();
    op.image[x] = uint32_t(y);
    op.matrix[x] = {v.re, v.im};
  }
  return op;
}

// ---------------------------------------------------------------------------
// noise (circuit.rs:98-147)
// ---------------------------------------------------------------------------
namespace {
struct ErrTerm {
  double p;
  int x, z;
};
std::vector<ErrTerm> noise_terms(const NoiseIR& n) {
  switch (n.kind) {
    case NoiseKind::XError: return {{n.p[0], 1, 0}};
    case NoiseKind::YError: return {{n.p[0], 1, 1}};
    case NoiseKind::ZError: return {{n.p[0], 0, 1}};
    case NoiseKind::PauliChannel1: return {{n.p[0], 1, 0}, {n.p[1], 1, 1}, {n.p[2], 0, 1}};
    case NoiseKind::Depolarize1: return {{n.p[0] / 3.0, 1, 0}, {n.p[0] / 3.0, 1, 1}, {n.p[0] / 3.0, 0, 1}};
    case NoiseKind::Depolarize2: {
      std::vector<ErrTerm> v;
      for (int k = 1; k < 16; ++k) v.push_back({n.p[0] / 15.0, k & 3, k >> 2});
      return v;
    }
  }
  return {};
}
}  // namespace

std::string NoiseIR::text() const {
  switch (kind) {
    case NoiseKind::XError: return "X_ERROR(" + fmt_f64(p[0]) + ")";
    case NoiseKind::YError: return "Y_ERROR(" + fmt_f64(p[0]) + ")";
    case NoiseKind::ZError: return "Z_ERROR(" + fmt_f64(p[0]) + ")";
    case NoiseKind::PauliChannel1: return "PAULI_CHANNEL_1(" + fmt_f64(p[0]) + "," + fmt_f64(p[1]) + "," + fmt_f64(p[2]) + ")";
    case NoiseKind::Depolarize1: return "DEPOLARIZE1(" + fmt_f64(p[0]) + ")";
    case NoiseKind::Depolarize2: return "DEPOLARIZE2(" + fmt_f64(p[0]) + ")";
  }
  return "?";
}

bool NoiseIR::valid() const {
  double s = 0;
  for (auto& t : noise_terms(*this)) {
    if (!(t.p >= 0.0 && t.p <= 1.0)) return false;
    s += t.p;
  }
  return s <= 1.0 + 1e-12;
}

int NoiseIR::sample(ncsim_rng& rng) const {
  double u = rng.f64();
  for (auto& t : noise_terms(*this)) {
    if (u < t.p) return t.x | (t.z << 8);
    u -= t.p;
  }
  return -1;
}

// ---------------------------------------------------------------------------
// circuits (circuit.rs:459-728)
// ---------------------------------------------------------------------------
static PhasePolyIR parse_poly(uint32_t nvars, const std::vector<std::string>& parts, size_t from, size_t to) {
  PhasePolyIR p;
  p.nvars = nvars;
  uint64_t bits, cst;
  if (to < from + 2 || !to_u64(parts[from], bits) || !to_u64(parts[from + 1], cst))
    throw parse_error("phase polynomial needs bits;constant");
  if (bits < 1 || bits > 32) throw Error(NCSIM_ERR_INVALID, "phase bits must be in 1..=32");
  p.bits = uint32_t(bits);
  p.constant = cst & mask_bits(p.bits);
  for (size_t i = from + 2; i < to; ++i) {
    auto ct = split_on(parts[i], ':');
    int64_t c;
    if (ct.size() != 2 || !to_i64(ct[0], c)) throw parse_error("bad term '" + parts[i] + "'");
    std::vector<uint64_t> pars;
    for (auto& m : split_on(ct[1], ',')) {
      uint64_t v;
      if (!to_u64(m, v)) throw parse_error("bad parity '" + m + "'");
      pars.push_back(v);
    }
    p.parities.push_back(pars);
    p.coeffs.push_back(uint64_t(emod(c, int64_t(mask_bits(p.bits)) + 1)));
  }
  return p;
}

GateIR parse_gate_token(const std::string& tok, uint32_t nq) {
  std::string name, inner;
  std::vector<std::string> args;
  size_t lp = tok.find('(');
  if (lp == std::string::npos) {
    name = upcase(tok);
  } else {
    name = upcase(tok.substr(0, lp));
    size_t rp = tok.rfind(')');
    if (rp == std::string::npos || rp < lp) throw parse_error("missing ')' in " + tok);
    inner = tok.substr(lp + 1, rp - lp - 1);
    for (auto& a : split_on(inner, ',')) args.push_back(strip(a));
  }
  static const std::map<std::string, GateKind> named = {
      {"I", GateKind::I}, {"X", GateKind::X}, {"Y", GateKind::Y}, {"Z", GateKind::Z}, {"H", GateKind::H},
      {"S", GateKind::S}, {"S_DAG", GateKind::Sdg}, {"SQRT_X", GateKind::SqrtX}, {"SQRT_X_DAG", GateKind::SqrtXdg},
      {"SQRT_Y", GateKind::SqrtY}, {"SQRT_Y_DAG", GateKind::SqrtYdg}, {"T", GateKind::T}, {"T_DAG", GateKind::Tdg},
      {"CX", GateKind::Cx}, {"CNOT", GateKind::Cx}, {"CY", GateKind::Cy}, {"CZ", GateKind::Cz},
      {"SWAP", GateKind::Swap}, {"CS", GateKind::Cs}, {"CS_DAG", GateKind::Csdg}, {"CCZ", GateKind::Ccz},
      {"CCX", GateKind::Ccx}, {"TOFFOLI", GateKind::Ccx}};
  GateIR g;
  auto it = named.find(name);
  if (it != named.end()) {
    g.kind = it->second;
    return g;
  }
  auto int_arg = [&](size_t i) {
    int64_t v;
    if (i >= args.size() || !to_i64(args[i], v)) throw parse_error(name + " needs integer argument " + std::to_string(i + 1));
    return v;
  };
  if (name == "PHASE" || name == "CPHASE") {
    g.kind = name == "PHASE" ? GateKind::Phase : GateKind::CPhase;
    g.pk = int_arg(0);
    int64_t b = int_arg(1);
    if (b < 1 || b > 32) throw Error(NCSIM_ERR_INVALID, "phase bits must be in 1..=32");
    g.pbits = uint32_t(b);
    return g;
  }
  if (name == "RX" || name == "RY" || name == "RZ") {
    g.kind = name == "RX" ? GateKind::Rx : name == "RY" ? GateKind::Ry : GateKind::Rz;
    if (args.empty() || !to_f64(args[0], g.theta)) throw parse_error(name + " needs a numeric argument");
    return g;
  }
  if (name == "DIAG") {
    auto parts = split_on(inner, ';');
    g.kind = GateKind::Diagonal;
    g.poly = parse_poly(nq, parts, 0, parts.size());
    return g;
  }
  if (name == "MONOMIAL") {
    auto parts = split_on(inner, ';');
    if (parts.size() < 5) throw parse_error("MONOMIAL(rows;shift;bits;constant;terms...;s2,phase,bits)");
    g.kind = GateKind::Monomial;
    MonomialIR& m = g.mono;
    m.k = nq;
    for (auto& r : split_on(parts[0], ',')) {
      uint64_t v;
      if (!to_u64(r, v)) throw parse_error("bad MONOMIAL row '" + r + "'");
      m.rows.push_back(v & mask_bits(nq));
    }
    if (m.rows.size() != nq) throw parse_error("MONOMIAL rows do not match its qubits");
    if (!to_u64(parts[1], m.shift)) throw parse_error("bad MONOMIAL shift");
    m.shift &= mask_bits(nq);
    m.phase = parse_poly(nq, parts, 2, parts.size() - 1);
    auto sc = split_on(parts.back(), ',');
    int64_t s2, sp, sb;
    if (sc.size() != 3 || !to_i64(sc[0], s2) || !to_i64(sc[1], sp) || !to_i64(sc[2], sb) || sb < 0 || sb > 62)
      throw parse_error("bad MONOMIAL scalar");
    m.scalar = Phase::make(int32_t(s2), sp, uint32_t(sb));
    if (gf2_rank_of(m.rows) != nq) throw Error(NCSIM_ERR_INVALID, "monomial gate: singular affine map");
    return g;
  }
  throw parse_error("unknown instruction '" + name + "'");
}

uint64_t ncsim_circuit_num_gates_impl(const ncsim_circuit& c);

}  // namespace ncsim

uint64_t ncsim_circuit::num_gates() const {
  uint64_t k = 0;
  for (auto& o : ops) k += o.kind == ncsim::OpKind::Gate;
  return k;
}
uint64_t ncsim_circuit::num_measurements() const {
  uint64_t k = 0;
  for (auto& o : ops) k += o.kind == ncsim::OpKind::Measure;
  return k;
}

std::string ncsim_circuit::text() const {
  using namespace ncsim;
  std::string s = "QUBITS " + std::to_string(n) + "\n";
  for (auto& o : ops) {
    switch (o.kind) {
      case OpKind::Gate:
        s += o.gate.text();
        for (uint32_t q : o.qubits) s += " " + std::to_string(q);
        break;
      case OpKind::Measure: {
        const auto& st = o.sites;
        static const char letters[] = "IXZY";
        if (st.sites.size() == 1 && st.phase == 0) {
          s += std::string("M") + letters[st.sites[0].second] + " " + std::to_string(st.sites[0].first);
        } else {
          static const char* pre[] = {"", "i*", "-", "-i*"};
          std::string body;
          for (auto& t : st.sites) {
            if (!body.empty()) body += "*";
            body += letters[t.second];
            body += std::to_string(t.first);
          }
          if (body.empty()) {
            static const char* sc[] = {"1", "i", "-1", "-i"};
            body = sc[st.phase & 3];
          } else {
            body = pre[st.phase & 3] + body;
          }
          s += "MPP " + body;
        }
        break;
      }
      case OpKind::Reset: s += "R " + std::to_string(o.qubits[0]); break;
      case OpKind::Noise:
        s += o.noise.text();
        for (uint32_t q : o.qubits) s += " " + std::to_string(q);
        break;
      case OpKind::Detector:
        s += "DETECTOR";
        for (uint64_t k : o.lookback) s += " rec[-" + std::to_string(k) + "]";
        break;
      case OpKind::Observable:
        s += "OBSERVABLE_INCLUDE(" + std::to_string(o.index) + ")";
        for (uint64_t k : o.lookback) s += " rec[-" + std::to_string(k) + "]";
        break;
      case OpKind::Tick: s += "TICK"; break;
    }
    s += "\n";
  }
  return s;
}

namespace ncsim {

ncsim_circuit parse_circuit(const std::string& text) {
  struct Line {
    size_t ln;
    std::vector<std::string> toks;
  };
  auto at = [](size_t ln, const std::string& m) { return parse_error("line " + std::to_string(ln + 1) + ": " + m); };
  std::vector<Line> lines;
  int64_t declared = -1;
  {
    size_t ln = 0, start = 0;
    while (start <= text.size()) {
      size_t e = text.find('\n', start);
      if (e == std::string::npos) e = text.size();
      std::string line = text.substr(start, e - start);
      size_t hash = line.find('#');
      if (hash != std::string::npos) line = line.substr(0, hash);
      std::istringstream is(line);
      Line L{ln, {}};
      std::string t;
      while (is >> t) L.toks.push_back(t);
      if (!L.toks.empty()) {
        if (upcase(L.toks[0]) == "QUBITS") {
          uint64_t v;
          if (L.toks.size() < 2 || !to_u64(L.toks[1], v)) throw at(ln, "QUBITS n");
          declared = int64_t(v);
        } else {
          lines.push_back(std::move(L));
        }
      }
      ++ln;
      start = e + 1;
    }
  }
  // first pass: instruction kinds, qubit lists and the register size
  struct Parsed {
    size_t ln;
    std::string head, name;
    std::vector<uint32_t> qs;
    std::vector<std::string> mpp;
    std::vector<uint64_t> recs;
  };
  std::vector<Parsed> ps;
  uint64_t max_q = 0;
  for (auto& L : lines) {
    Parsed p;
    p.ln = L.ln;
    p.head = L.toks[0];
    size_t lp = p.head.find('(');
    p.name = upcase(lp == std::string::npos ? p.head : p.head.substr(0, lp));
    if (p.name == "MPP") {
      for (size_t i = 1; i < L.toks.size(); ++i) {
        PauliSites q;
        try {
          q = parse_pauli_sites(L.toks[i], -1);
        } catch (const Error& e) {
          throw at(L.ln, e.what());
        }
        max_q = std::max<uint64_t>(max_q, q.n);
        p.mpp.push_back(L.toks[i]);
      }
    } else if (p.name == "DETECTOR" || p.name == "OBSERVABLE_INCLUDE") {
      for (size_t i = 1; i < L.toks.size(); ++i) {
        const std::string& t = L.toks[i];
        uint64_t k;
        if (t.rfind("rec[-", 0) != 0 || t.back() != ']' || !to_u64(t.substr(5, t.size() - 6), k))
          throw at(L.ln, "bad target '" + t + "' (expected rec[-k])");
        p.recs.push_back(k);
      }
    } else if (p.name == "TICK") {
    } else {
      for (size_t i = 1; i < L.toks.size(); ++i) {
        uint64_t q;
        if (!to_u64(L.toks[i], q) || q >= MAX_CIRCUIT_QUBITS) throw at(L.ln, "bad qubit '" + L.toks[i] + "'");
        p.qs.push_back(uint32_t(q));
        max_q = std::max<uint64_t>(max_q, q + 1);
      }
    }
    ps.push_back(std::move(p));
  }
  const uint64_t n = declared >= 0 ? uint64_t(declared) : max_q;
  if (n < max_q) throw parse_error("QUBITS " + std::to_string(n) + " but qubit " + std::to_string(max_q - 1) + " is used");
  if (n > MAX_CIRCUIT_QUBITS) throw parse_error("registers of more than " + std::to_string(MAX_CIRCUIT_QUBITS) + " qubits");
  ncsim_circuit c;
  c.n = uint32_t(n);
  uint64_t measured = 0;
  auto push_gate = [&](size_t ln, const GateIR& g, const std::vector<uint32_t>& qs) {
    OpIR o;
    o.kind = OpKind::Gate;
    o.gate = g;
    o.qubits = qs;
    try {
      if (c.n <= 64) {
        o.lowered = lower_gate(g, qs, c.n);
      } else {
        // wider than 64 qubits: the same checks, the gate lowered on its own qubits (local
        // qubit j is qs[j]; the wide sparse form maps them back)
        std::vector<uint32_t> local(qs.size());
        for (size_t i = 0; i < qs.size(); ++i) {
          if (qs[i] >= c.n) throw qubit_out_of_range(qs[i], c.n);
          for (size_t j = 0; j < i; ++j)
            if (qs[j] == qs[i]) throw duplicate_qubit(qs[i]);
          local[i] = uint32_t(i);
        }
        if (qs.size() <= 64) o.lowered = lower_gate(g, local, uint32_t(qs.size()));
        else if (qs.size() != g.arity()) throw arity_error(g.text(), g.arity(), qs.size());
      }
    } catch (const Error& e) {
      throw Error(e.code == NCSIM_ERR_PARSE ? e.code : NCSIM_ERR_PARSE, "line " + std::to_string(ln + 1) + ": " + e.what());
    }
    c.ops.push_back(std::move(o));
  };
  for (auto& p : ps) {
    const std::string& nm = p.name;
    if (nm == "M" || nm == "MZ" || nm == "MX" || nm == "MY") {
      char letter = nm == "MX" ? 'X' : nm == "MY" ? 'Y' : 'Z';
      for (uint32_t q : p.qs) {
        OpIR o;
        o.kind = OpKind::Measure;
        o.sites.n = c.n;
        o.sites.sites = {{q, uint8_t(letter == 'X' ? 1 : letter == 'Z' ? 2 : 3)}};
        o.pauli.n = c.n;
        if (c.n <= 64) set_letter(o.pauli, q, letter);
        c.ops.push_back(o);
        ++measured;
      }
    } else if (nm == "MPP") {
      for (auto& t : p.mpp) {
        OpIR o;
        o.kind = OpKind::Measure;
        try {
          o.sites = parse_pauli_sites(t, int64_t(c.n));
        } catch (const Error& e) {
          throw at(p.ln, e.what());
        }
        if (!o.sites.hermitian()) throw at(p.ln, "measured operator " + t + " is not Hermitian");
        o.pauli.n = c.n;
        if (c.n <= 64) o.pauli = pauli_from_sites(o.sites);
        c.ops.push_back(o);
        ++measured;
      }
    } else if (nm == "R") {
      for (uint32_t q : p.qs) {
        OpIR o;
        o.kind = OpKind::Reset;
        o.qubits = {q};
        c.ops.push_back(o);
      }
    } else if (nm == "X_ERROR" || nm == "Y_ERROR" || nm == "Z_ERROR" || nm == "DEPOLARIZE1" || nm == "DEPOLARIZE2" ||
               nm == "PAULI_CHANNEL_1") {
      NoiseIR nz;
      nz.kind = nm == "X_ERROR" ? NoiseKind::XError : nm == "Y_ERROR" ? NoiseKind::YError : nm == "Z_ERROR" ? NoiseKind::ZError
              : nm == "DEPOLARIZE1" ? NoiseKind::Depolarize1 : nm == "DEPOLARIZE2" ? NoiseKind::Depolarize2
                                                                                  : NoiseKind::PauliChannel1;
      size_t lp = p.head.find('('), rp = p.head.rfind(')');
      if (lp == std::string::npos) throw at(p.ln, nm + " needs a numeric argument");
      if (rp == std::string::npos || rp < lp) throw at(p.ln, "missing ')' in " + p.head);
      auto args = split_on(p.head.substr(lp + 1, rp - lp - 1), ',');
      size_t need = nz.kind == NoiseKind::PauliChannel1 ? 3 : 1;
      for (size_t i = 0; i < need; ++i)
        if (i >= args.size() || !to_f64(args[i], nz.p[i]))
          throw at(p.ln, nz.kind == NoiseKind::PauliChannel1 ? "PAULI_CHANNEL_1 needs three probabilities"
                                                             : nm + " needs a numeric argument");
      const uint32_t k = nz.arity();
      if (p.qs.size() % k) throw at(p.ln, nz.text() + " takes groups of " + std::to_string(k) + " qubits");
      if (!nz.valid()) throw at(p.ln, nz.text() + " is not a probability distribution");
      for (size_t i = 0; i < p.qs.size(); i += k) {
        OpIR o;
        o.kind = OpKind::Noise;
        o.noise = nz;
        o.qubits.assign(p.qs.begin() + i, p.qs.begin() + i + k);
        if (k == 2 && o.qubits[0] == o.qubits[1]) throw at(p.ln, "qubit " + std::to_string(o.qubits[0]) + " listed twice");
        c.ops.push_back(o);
      }
    } else if (nm == "DETECTOR" || nm == "OBSERVABLE_INCLUDE") {
      OpIR o;
      o.kind = nm == "DETECTOR" ? OpKind::Detector : OpKind::Observable;
      o.lookback = p.recs;
      for (uint64_t k : p.recs)
        if (k == 0 || k > measured) throw at(p.ln, "rec[-" + std::to_string(k) + "] with " + std::to_string(measured) + " measurements so far");
      if (o.kind == OpKind::Observable) {
        size_t lp = p.head.find('(');
        int64_t idx;
        if (lp == std::string::npos || !to_i64(p.head.substr(lp + 1, p.head.rfind(')') - lp - 1), idx) || idx < 0)
          throw at(p.ln, "OBSERVABLE_INCLUDE needs integer argument 1");
        o.index = uint64_t(idx);
      }
      c.ops.push_back(o);
    } else if (nm == "TICK") {
      OpIR o;
      o.kind = OpKind::Tick;
      c.ops.push_back(o);
    } else {
      GateIR g;
      try {
        g = parse_gate_token(p.head, uint32_t(p.qs.size()));
      } catch (const Error& e) {
        throw at(p.ln, e.what());
      }
      if (g.kind == GateKind::Diagonal || g.kind == GateKind::Monomial) {
        push_gate(p.ln, g, p.qs);
        continue;
      }
      const uint32_t k = g.arity();
      if (k == 0 || p.qs.size() % k) throw at(p.ln, g.text() + " takes groups of " + std::to_string(k) + " qubits");
      for (size_t i = 0; i < p.qs.size(); i += k)
        push_gate(p.ln, g, std::vector<uint32_t>(p.qs.begin() + i, p.qs.begin() + i + k));
    }
  }
  return c;
}

}  // namespace ncsim
