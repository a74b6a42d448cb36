// Precision form, host side: planning, fusion, operand images, emulation.
#include "fused_plan.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>

namespace ncsim {
namespace fused {

namespace {

enum class GClass { Skip, Diag, Dense, Plain };

struct GInfo {
  GClass cls = GClass::Skip;
  std::vector<uint32_t> q;
  std::vector<CplxD> m;  // Dense: 2^k x 2^k row-major
  std::vector<CplxD> d;  // Diag: 2^k entries
  uint64_t mask = 0;
};

inline CplxD mul(CplxD a, CplxD b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline CplxD inv(CplxD a) {
  const double s = a.re * a.re + a.im * a.im;
  return {a.re / s, -a.im / s};
}
inline bool exactly_one(CplxD c) { return c.re == 1.0 && c.im == 0.0; }

GInfo classify(const OpIR& op) {
  GInfo g;
  if (op.kind == OpKind::Tick || op.kind == OpKind::Detector || op.kind == OpKind::Observable) return g;
  if (op.kind != OpKind::Gate) {
    g.cls = GClass::Plain;
    return g;
  }
  const LoweredOp& lo = op.lowered;
  g.q = lo.qubits;
  for (uint32_t q : g.q) g.mask |= uint64_t(1) << q;
  const size_t k = g.q.size(), d = size_t(1) << k;
  switch (lo.kind) {
    case LoweredKind::Nothing: g.cls = GClass::Skip; return g;
    case LoweredKind::PhasePoly:
    case LoweredKind::Pauli: g.cls = GClass::Plain; return g;
    case LoweredKind::Dense: {
      bool diag = true;
      for (size_t r = 0; r < d && diag; ++r)
        for (size_t c = 0; c < d; ++c)
          if (r != c && (lo.matrix[r * d + c].re != 0.0 || lo.matrix[r * d + c].im != 0.0)) {
            diag = false;
            break;
          }
      if (diag && k <= 3) {
        g.cls = GClass::Diag;
        for (size_t x = 0; x < d; ++x) g.d.push_back(lo.matrix[x * d + x]);
      } else if (k <= size_t(GROUP_QUBITS)) {
        g.cls = GClass::Dense;
        g.m = lo.matrix;
      } else {
        g.cls = GClass::Plain;
      }
      return g;
    }
    case LoweredKind::Monomial: {
      bool ident = true;
      for (size_t x = 0; x < d; ++x) ident &= lo.image[x] == x;
      if (ident && k <= 3) {
        g.cls = GClass::Diag;
        g.d = lo.matrix;
      } else if (k <= size_t(GROUP_QUBITS)) {
        g.cls = GClass::Dense;
        g.m.assign(d * d, CplxD{0, 0});
        for (size_t x = 0; x < d; ++x) g.m[size_t(lo.image[x]) * d + x] = lo.matrix[x];
      } else {
        g.cls = GClass::Plain;
      }
      return g;
    }
  }
  g.cls = GClass::Plain;
  return g;
}

// diag(d) over local bits -> product of (mask, c) terms: c_S = prod_{T in S} d[T]^{(-1)^{|S|-|T|}}
void diag_terms(const GInfo& g, std::vector<Term>& out) {
  const size_t k = g.q.size(), dsz = size_t(1) << k;
  for (size_t s = 0; s < dsz; ++s) {
    CplxD c{1.0, 0.0};
    for (size_t t = s;; t = (t - 1) & s) {
      const int sign = (__builtin_popcountll(s) - __builtin_popcountll(t)) & 1;
      c = mul(c, sign ? inv(g.d[t]) : g.d[t]);
      if (t == 0) break;
    }
    if (exactly_one(c)) continue;
    uint64_t m = 0;
    for (size_t j = 0; j < k; ++j)
      if ((s >> j) & 1) m |= uint64_t(1) << g.q[j];
    out.push_back({m, c});
  }
}

// An open fused group: a unitary over the local qubits q (bit j = q[j]).
struct Group {
  std::vector<uint32_t> q;
  std::vector<CplxD> u;  // 2^|q| square
  uint64_t mask = 0;
  bool open = false;

  void start() {
    q.clear();
    u.assign(1, CplxD{1.0, 0.0});
    mask = 0;
    open = true;
  }
  void add_qubit(uint32_t qb) {
    const size_t d = size_t(1) << q.size();
    std::vector<CplxD> nu(4 * d * d, CplxD{0, 0});
    // U (x) I on the new highest local bit
    for (size_t h = 0; h < 2; ++h)
      for (size_t r = 0; r < d; ++r)
        for (size_t c = 0; c < d; ++c) nu[(h * d + r) * (2 * d) + (h * d + c)] = u[r * d + c];
    u.swap(nu);
    q.push_back(qb);
    mask |= uint64_t(1) << qb;
  }
  int local_of(uint32_t qb) const {
    for (size_t j = 0; j < q.size(); ++j)
      if (q[j] == qb) return int(j);
    return -1;
  }
  // U <- G U for a dense gate G on (a subset of) the group's qubits
  void apply_dense(const std::vector<uint32_t>& gq, const std::vector<CplxD>& gm) {
    for (uint32_t qb : gq)
      if (local_of(qb) < 0) add_qubit(qb);
    const size_t d = size_t(1) << q.size(), k = gq.size(), gd = size_t(1) << k;
    std::vector<int> pos(k);
    uint64_t gmask = 0;
    for (size_t j = 0; j < k; ++j) pos[j] = local_of(gq[j]), gmask |= uint64_t(1) << pos[j];
    std::vector<CplxD> nu(d * d, CplxD{0, 0});
    for (size_t row = 0; row < d; ++row) {
      size_t a = 0;
      for (size_t j = 0; j < k; ++j) a |= ((row >> pos[j]) & 1) << j;
      const size_t rest = row & ~gmask;
      for (size_t b = 0; b < gd; ++b) {
        const CplxD gv = gm[a * gd + b];
        if (gv.re == 0.0 && gv.im == 0.0) continue;
        size_t src = rest;
        for (size_t j = 0; j < k; ++j) src |= ((b >> j) & 1) << pos[j];
        for (size_t c = 0; c < d; ++c) {
          const CplxD t = mul(gv, u[src * d + c]);
          nu[row * d + c].re += t.re;
          nu[row * d + c].im += t.im;
        }
      }
    }
    u.swap(nu);
  }
  void apply_diag(const std::vector<uint32_t>& gq, const std::vector<CplxD>& dg) {
    const size_t d = size_t(1) << q.size();
    std::vector<int> pos(gq.size());
    for (size_t j = 0; j < gq.size(); ++j) pos[j] = local_of(gq[j]);
    for (size_t row = 0; row < d; ++row) {
      size_t a = 0;
      for (size_t j = 0; j < gq.size(); ++j) a |= ((row >> pos[j]) & 1) << j;
      for (size_t c = 0; c < d; ++c) u[row * d + c] = mul(dg[a], u[row * d + c]);
    }
  }
};

std::vector<Term> merge_terms(const std::vector<Term>& in) {
  std::map<uint64_t, CplxD> acc;
  for (auto& t : in) {
    auto it = acc.find(t.mask);
    if (it == acc.end()) acc[t.mask] = t.c;
    else it->second = mul(it->second, t.c);
  }
  std::vector<Term> out;
  for (auto& kv : acc)
    if (!exactly_one(kv.second)) out.push_back({kv.first, kv.second});
  return out;
}

// d (on gate qubits gq) folded into an emitted unitary op: U <- D U
void fold_diag_into(FusedOp& op, const GInfo& d) {
  Group tmp;
  tmp.q = op.qubits;
  tmp.u = op.u;
  for (uint32_t q : op.qubits) tmp.mask |= uint64_t(1) << q;
  tmp.apply_diag(d.q, d.d);
  op.u.swap(tmp.u);
}

uint64_t qubit_mask(const std::vector<uint32_t>& qs) {
  uint64_t m = 0;
  for (uint32_t q : qs) m |= uint64_t(1) << q;
  return m;
}

// How the pass kernel can apply a term next to a unitary on the qubits gm:
// 0 as a phase of the whole column (no gate qubit in its mask), 1 as a sign
// on the rows of one gate qubit (a -1 conditioned on that qubit and column
// bits), 2 neither (a sweep of its own).
int term_relation(const Term& t, uint64_t gm) {
  const uint64_t gp = t.mask & gm;
  if (!gp) return 0;
  if (__builtin_popcountll(gp) == 1 && t.c.re == -1.0 && t.c.im == 0.0) return 1;
  return 2;
}

// Places a pass's elementwise terms.  Diagonal terms commute with each other
// and with every unitary whose qubits they do not share, so each term moves
// right to the gap before the first unitary that touches its qubits (or to the
// end of the pass); one whose qubits all lie in that unitary is multiplied
// into it (U <- U D, FP64), the rest gather in fewer gaps.  Each gap then holds
// up to three term ops in this order: the terms the previous unitary's
// read-back can apply, the ones that need a sweep of their own, and the ones
// the next unitary's split can apply.  Every gap with terms costs the kernel a
// per-amplitude phase or sign step, so fewer gaps mean fewer of them.
void place_terms(Pass& pass) {
  std::vector<FusedOp> us;
  std::vector<std::vector<Term>> gaps(1);  // gaps[i]: terms before unitary i; the last: after all
  for (FusedOp& op : pass.ops) {
    if (op.kind == 0) {
      us.push_back(std::move(op));
      gaps.emplace_back();
    } else {
      for (const Term& t : op.terms) gaps.back().push_back(t);
    }
  }
  const size_t nu = us.size();
  std::vector<uint64_t> gm(nu);
  for (size_t i = 0; i < nu; ++i) gm[i] = qubit_mask(us[i].qubits);
  std::vector<std::vector<Term>> placed(nu + 1);
  for (size_t i = 0; i <= nu; ++i)
    for (const Term& t : gaps[i]) {
      size_t j = i;
      while (j < nu && !(t.mask & gm[j])) ++j;
      if (j < nu && (t.mask & ~gm[j]) == 0) {
        // U <- U D: column c of U takes the phase when its local index holds every bit of the mask
        const std::vector<uint32_t>& q = us[j].qubits;
        uint32_t lm = 0;
        for (size_t b = 0; b < q.size(); ++b)
          if ((t.mask >> q[b]) & 1) lm |= 1u << b;
        const size_t d = size_t(1) << q.size();
        for (size_t c = 0; c < d; ++c)
          if ((uint32_t(c) & lm) == lm)
            for (size_t r = 0; r < d; ++r) us[j].u[r * d + c] = mul(us[j].u[r * d + c], t.c);
        continue;
      }
      placed[j].push_back(t);
    }
  pass.ops.clear();
  for (size_t i = 0; i <= nu; ++i) {
    std::vector<Term> post, sweep, pre;
    for (const Term& t : merge_terms(placed[i])) {
      if (i < nu && term_relation(t, gm[i]) < 2) pre.push_back(t);
      else if (i > 0 && term_relation(t, gm[i - 1]) < 2) post.push_back(t);
      else sweep.push_back(t);
    }
    for (std::vector<Term>* ts : {&post, &sweep, &pre}) {
      if (ts->empty()) continue;
      FusedOp op;
      op.kind = 1;
      op.terms = std::move(*ts);
      pass.ops.push_back(std::move(op));
    }
    if (i < nu) pass.ops.push_back(std::move(us[i]));
  }
}

// Builds one pass's program.  Diagonal gates are folded into a unitary on
// their qubits whenever the order allows: into the most recent unitary that
// touches them (everything applied to those qubits after it is diagonal, and
// diagonals commute), or into the unitary that a later gate on the same
// qubits opens; only the rest become elementwise terms.  Global phases are
// folded into any unitary of the pass.
struct PassBuilder {
  uint64_t window = 0;
  Pass pass;
  Group g;
  std::vector<GInfo> pending;  // diagonal gates waiting, in order
  uint64_t pending_mask = 0;
  int emitted_unitaries = 0;
  size_t term_count = 0;
  CplxD global{1.0, 0.0};

  void emit_group() {
    if (!g.open) return;
    // pad to exactly 5 window qubits (U (x) I) with the highest free window
    // qubits: the lowest tile bits then stay column bits, so the 32 columns a
    // warp reads spread over all shared-memory banks
    for (int b = 63; b >= 0 && g.q.size() < size_t(GROUP_QUBITS); --b)
      if (((window >> b) & 1) && g.local_of(uint32_t(b)) < 0) g.add_qubit(uint32_t(b));
    FusedOp op;
    op.kind = 0;
    op.qubits = g.q;
    op.u = g.u;
    pass.ops.push_back(std::move(op));
    ++emitted_unitaries;
    g.open = false;
  }
  void emit_terms(const std::vector<GInfo>& ds) {
    std::vector<Term> t;
    for (const GInfo& d : ds) diag_terms(d, t);
    std::vector<Term> merged = merge_terms(t);
    FusedOp op;
    op.kind = 1;
    for (const Term& tm : merged) {
      if (tm.mask == 0) global = mul(global, tm.c);
      else op.terms.push_back(tm);
    }
    term_count += op.terms.size();
    if (!op.terms.empty()) pass.ops.push_back(std::move(op));
  }
  void emit_pending() {
    if (pending.empty()) return;
    emit_terms(pending);
    pending.clear();
    pending_mask = 0;
  }
  // worst-case number of terms the pending gates could add
  size_t pending_term_bound() const {
    size_t s = 0;
    for (const GInfo& d : pending) s += size_t(1) << d.q.size();
    return s;
  }
  // false: the gate does not fit this pass's limits (the caller cuts here)
  bool add(const GInfo& gi, int maxk) {
    if (gi.cls == GClass::Diag) {
      // backward: the most recent unitary touching these qubits
      if (g.open && (g.mask & gi.mask)) {
        if ((gi.mask & ~g.mask) == 0) {
          g.apply_diag(gi.q, gi.d);
          return true;
        }
        // the open group takes the gate's other window qubits along while it has room:
        // the gate becomes part of the unitary instead of a term that blocks later
        // gates on those qubits
        if ((gi.mask & ~window) == 0 && !(gi.mask & pending_mask) &&
            __builtin_popcountll(g.mask | gi.mask) <= maxk) {
          for (uint32_t q : gi.q)
            if (g.local_of(q) < 0) g.add_qubit(q);
          g.apply_diag(gi.q, gi.d);
          return true;
        }
      } else {
        for (size_t i = pass.ops.size(); i-- > 0;) {
          if (pass.ops[i].kind != 0) continue;
          const uint64_t m = qubit_mask(pass.ops[i].qubits);
          if (!(m & gi.mask)) continue;
          if ((gi.mask & ~m) == 0) {
            fold_diag_into(pass.ops[i], gi);
            return true;
          }
          break;
        }
      }
      if (term_count + pending_term_bound() + (size_t(1) << gi.q.size()) > size_t(MAX_TERMS)) return false;
      if (pass.ops.size() + 3 > size_t(MAX_OPS)) return false;
      pending.push_back(gi);
      pending_mask |= gi.mask;
      return true;
    }
    if (g.open && __builtin_popcountll(g.mask | gi.mask) <= maxk && !(gi.mask & pending_mask)) {
      g.apply_dense(gi.q, gi.m);
      return true;
    }
    // a new group
    if (emitted_unitaries + (g.open ? 1 : 0) + 1 > MAX_UNITARIES) return false;
    if (pass.ops.size() + 3 > size_t(MAX_OPS)) return false;
    emit_group();
    // forward: waiting diagonals on this gate's qubits open the new group
    // (they come after every emitted op on their qubits and before this gate)
    std::vector<GInfo> fold, keep;
    for (const GInfo& d : pending) ((d.mask & ~gi.mask) == 0 ? fold : keep).push_back(d);
    if (!keep.empty()) emit_terms(keep);
    pending.clear();
    pending_mask = 0;
    g.start();
    for (uint32_t q : gi.q) g.add_qubit(q);
    for (const GInfo& d : fold) g.apply_diag(d.q, d.d);
    g.apply_dense(gi.q, gi.m);
    return true;
  }
  Pass finish(uint32_t n) {
    emit_group();
    emit_pending();
    // the global phase goes into a unitary when the pass has one
    if (!exactly_one(global)) {
      bool folded = false;
      for (auto& op : pass.ops)
        if (op.kind == 0) {
          for (auto& e : op.u) e = mul(global, e);
          folded = true;
          break;
        }
      if (!folded) {
        FusedOp op;
        op.kind = 1;
        op.terms.push_back({0, global});
        pass.ops.push_back(std::move(op));
        ++term_count;
      }
    }
    place_terms(pass);
    // window: exactly TILE_BITS qubits, ascending
    uint64_t w = window;
    for (uint32_t b = 0; b < n && __builtin_popcountll(w) < TILE_BITS; ++b) w |= uint64_t(1) << b;
    pass.window.clear();
    for (uint32_t b = 0; b < 64; ++b)
      if ((w >> b) & 1) pass.window.push_back(b);
    pass.unitaries = emitted_unitaries;
    return std::move(pass);
  }
};

// Passes for a run of fusable gates, in dependency order.
// lookahead: each pass's window may also be grown qubit by qubit (the one that
// lets the most dense gates through), keeping it when it lets more through than
// the first-come window.
void plan_run(const std::vector<GInfo>& gs, uint32_t n, int maxk, bool lookahead_windows, std::vector<Pass>& out,
              Plan& stats) {
  std::vector<size_t> remaining(gs.size());
  for (size_t i = 0; i < gs.size(); ++i) remaining[i] = i;
  const uint64_t low = (uint64_t(1) << LOW_BITS) - 1;
  // the dense gates a fixed window lets through (gates behind a blocked qubit wait)
  auto dense_through = [&](uint64_t W) {
    uint64_t blocked = 0;
    size_t dense = 0;
    for (size_t i : remaining) {
      const GInfo& g = gs[i];
      if (g.mask & blocked) blocked |= g.mask;
      else if (g.cls == GClass::Diag) continue;
      else if ((g.mask & ~W) == 0) ++dense;
      else blocked |= g.mask;
    }
    return dense;
  };
  while (!remaining.empty()) {
    // the window, first come first served: qubits of the gates in circuit order
    uint64_t W = low, blocked = 0;
    for (size_t i : remaining) {
      const GInfo& g = gs[i];
      if (g.mask & blocked) blocked |= g.mask;
      else if (g.cls == GClass::Diag) continue;
      else if (__builtin_popcountll(W | g.mask) <= TILE_BITS) W |= g.mask;
      else blocked |= g.mask;
    }
    for (uint32_t b = 0; b < n && __builtin_popcountll(W) < TILE_BITS; ++b) W |= uint64_t(1) << b;
    // and a window grown one qubit at a time, each time the qubit that lets the most
    // dense gates through; the better of the two is taken
    if (lookahead_windows) {
      uint64_t G = low;
      while (__builtin_popcountll(G) < TILE_BITS) {
        size_t best = 0;
        uint32_t bq = n;
        for (uint32_t q = 0; q < n; ++q) {
          if ((G >> q) & 1) continue;
          const size_t d = dense_through(G | (uint64_t(1) << q));
          if (bq == n || d > best) best = d, bq = q;
        }
        G |= uint64_t(1) << bq;
      }
      if (dense_through(G) > dense_through(W)) W = G;
    }
    // the gates the window takes, in order
    blocked = 0;
    std::vector<size_t> inc, rest;
    for (size_t i : remaining) {
      const GInfo& g = gs[i];
      if ((g.mask & blocked) || (g.cls != GClass::Diag && (g.mask & ~W))) {
        blocked |= g.mask;
        rest.push_back(i);
      } else {
        inc.push_back(i);
      }
    }
    // fuse; gates past the pass's limits go back (they depend on nothing left behind)
    PassBuilder pb;
    pb.window = W;
    size_t taken = 0;
    for (; taken < inc.size(); ++taken)
      if (!pb.add(gs[inc[taken]], maxk)) break;
    if (taken == 0) throw Error(NCSIM_ERR_INVALID, "fusion planner made no progress");
    Pass p = pb.finish(n);
    stats.unitaries += uint64_t(p.unitaries);
    for (auto& op : p.ops) stats.terms += op.terms.size();
    out.push_back(std::move(p));
    std::vector<size_t> back(inc.begin() + taken, inc.end());
    std::vector<size_t> merged;
    std::merge(rest.begin(), rest.end(), back.begin(), back.end(), std::back_inserter(merged));
    remaining.swap(merged);
  }
}

}  // namespace

Plan make_plan(const ncsim_circuit& c, uint32_t max_fuse) {
  if (c.n < uint32_t(TILE_BITS)) throw Error(NCSIM_ERR_UNSUPPORTED, "the fused form needs at least 12 qubits");
  const int maxk = int(std::min<uint32_t>(std::max<uint32_t>(max_fuse, 1), GROUP_QUBITS));
  Plan p;
  p.n = c.n;
  std::vector<GInfo> run;
  auto flush = [&] {
    if (run.empty()) return;
    Segment s;
    s.fused = true;
    // Both window rules, and the cheaper plan by the pass kernel's measured cost:
    // a pass costs about as much as 1.36 unitaries (its streaming), so fewer passes
    // win only when they do not add more unitaries than that.
    Plan pa, pb;
    std::vector<Pass> a, b;
    plan_run(run, c.n, maxk, false, a, pa);
    plan_run(run, c.n, maxk, true, b, pb);
    auto cost = [](const std::vector<Pass>& v, const Plan& st) {
      return 1.36 * double(v.size()) + double(st.unitaries) + 1e-4 * double(st.terms);
    };
    const bool take_b = cost(b, pb) < cost(a, pa);
    s.passes = take_b ? std::move(b) : std::move(a);
    const Plan& ps = take_b ? pb : pa;
    p.unitaries += ps.unitaries;
    p.terms += ps.terms;
    p.passes += s.passes.size();
    p.segments.push_back(std::move(s));
    run.clear();
  };
  for (size_t i = 0; i < c.ops.size(); ++i) {
    const OpIR& op = c.ops[i];
    if (op.kind == OpKind::Gate) ++p.source_gates;
    GInfo g = classify(op);
    if (g.cls == GClass::Skip) continue;
    if (g.cls == GClass::Plain) {
      flush();
      Segment s;
      s.fused = false;
      s.op = i;
      p.segments.push_back(std::move(s));
      continue;
    }
    run.push_back(std::move(g));
  }
  flush();
  return p;
}

// ---------------------------------------------------------------------------
uint16_t bf16_bits(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return uint16_t(u >> 16);  // inf / nan (never used)
  const uint32_t rounding = 0x7fffu + ((u >> 16) & 1u);             // to nearest, ties to even
  return uint16_t((u + rounding) >> 16);
}

float bf16_value(uint16_t b) {
  const uint32_t u = uint32_t(b) << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

void build_operand_image(const std::vector<CplxD>& u, uint8_t* out) {
  // R[n][k]: output n = 2 row + (0 real, 1 imaginary), so the accumulator holds each row's
  // real and imaginary parts in adjacent columns; k < 32 real inputs, k >= 32 imaginary
  std::memset(out, 0, 16384);
  uint16_t* hi = reinterpret_cast<uint16_t*>(out);
  uint16_t* lo = reinterpret_cast<uint16_t*>(out + 8192);
  for (uint32_t n = 0; n < 64; ++n)
    for (uint32_t k = 0; k < 64; ++k) {
      const CplxD e = u[(n >> 1) * 32 + (k & 31)];
      const bool im_out = n & 1;
      double r;
      if (!im_out && k < 32) r = e.re;
      else if (!im_out) r = -e.im;
      else if (k < 32) r = e.im;
      else r = e.re;
      const float rf = float(r);
      const uint16_t h = bf16_bits(rf);
      const uint16_t l = bf16_bits(float(r - double(bf16_value(h))));
      const uint32_t off = sw128_offset(n, k >> 3) + (k & 7) * 2;
      hi[off / 2] = h;
      lo[off / 2] = l;
    }
}

// a lowered gate on host amplitudes (the plain segments of the emulation)
static void apply_lowered_host(const LoweredOp& op, std::vector<CplxD>& a, uint32_t n) {
  const uint64_t len = uint64_t(1) << n;
  const size_t k = op.qubits.size();
  auto local = [&](uint64_t i) {
    uint64_t x = 0;
    for (size_t j = 0; j < k; ++j) x |= ((i >> op.qubits[j]) & 1) << j;
    return x;
  };
  auto with_local = [&](uint64_t i, uint64_t y) {
    for (size_t j = 0; j < k; ++j) i = (i & ~(uint64_t(1) << op.qubits[j])) | (((y >> j) & 1) << op.qubits[j]);
    return i;
  };
  std::vector<CplxD> out(a.size(), CplxD{0, 0});
  switch (op.kind) {
    case LoweredKind::Nothing: return;
    case LoweredKind::Pauli:
      for (uint64_t c = 0; c < len; ++c) {
        const int kk = int(op.phase + 2 * __builtin_popcountll(op.z & c)) & 3;
        static const CplxD ip[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
        out[c ^ op.x] = mul(ip[kk], a[c]);
      }
      break;
    case LoweredKind::PhasePoly:
      for (uint64_t i = 0; i < len; ++i) {
        uint64_t f = op.poly.constant;
        for (size_t t = 0; t + 1 < op.poly.term_start.size(); ++t) {
          bool all = true;
          for (uint32_t l = op.poly.term_start[t]; l < op.poly.term_start[t + 1]; ++l)
            all &= bool(__builtin_popcountll(op.poly.parities[l] & i) & 1);
          if (all) f += op.poly.coeffs[t];
        }
        f &= (uint64_t(1) << op.poly.bits) - 1;
        Cd r = root_value(int64_t(f), op.poly.bits);
        CplxD c = op.poly.root_table.empty() ? mul(op.poly.scalar, CplxD{r.re, r.im}) : op.poly.root_table[f];
        out[i] = mul(c, a[i]);
      }
      break;
    case LoweredKind::Monomial:
      for (uint64_t i = 0; i < len; ++i) {
        const uint64_t x = local(i);
        out[with_local(i, op.image[x])] = mul(op.matrix[x], a[i]);
      }
      break;
    case LoweredKind::Dense: {
      const size_t d = size_t(1) << k;
      for (uint64_t i = 0; i < len; ++i) {
        const uint64_t x = local(i);
        for (size_t y = 0; y < d; ++y) {
          CplxD m = mul(op.matrix[y * d + x], a[i]);
          CplxD& o = out[with_local(i, y)];
          o.re += m.re;
          o.im += m.im;
        }
      }
      break;
    }
  }
  a.swap(out);
}

void emulate(const Plan& p, const ncsim_circuit& c, std::vector<CplxD>& a) {
  const uint64_t len = uint64_t(1) << p.n;
  for (const Segment& s : p.segments) {
    if (!s.fused) {
      const OpIR& op = c.ops[s.op];
      if (op.kind != OpKind::Gate) throw Error(NCSIM_ERR_UNSUPPORTED, "emulation covers gates only");
      apply_lowered_host(op.lowered, a, p.n);
      continue;
    }
    for (const Pass& ps : s.passes) {
      uint64_t wmask = 0;
      for (uint32_t b : ps.window) wmask |= uint64_t(1) << b;
      const uint64_t ntiles = len >> TILE_BITS;
      std::vector<CplxD> t(size_t(1) << TILE_BITS);
      for (uint64_t tile = 0; tile < ntiles; ++tile) {
        // base: tile bits deposited outside the window
        uint64_t base = 0;
        for (uint32_t b = 0, j = 0; b < p.n; ++b)
          if (!((wmask >> b) & 1)) base |= ((tile >> j++) & 1) << b;
        auto gidx = [&](uint32_t e) {
          uint64_t g = base;
          for (int j = 0; j < TILE_BITS; ++j) g |= uint64_t((e >> j) & 1) << ps.window[j];
          return g;
        };
        for (uint32_t e = 0; e < t.size(); ++e) t[e] = a[gidx(e)];
        for (const FusedOp& op : ps.ops) {
          if (op.kind == 1) {
            for (uint32_t e = 0; e < t.size(); ++e) {
              const uint64_t gi = gidx(e);
              for (const Term& tm : op.terms)
                if ((gi & tm.mask) == tm.mask) t[e] = mul(tm.c, t[e]);
            }
            continue;
          }
          int pos[GROUP_QUBITS];
          uint32_t gt = 0;
          for (int j = 0; j < GROUP_QUBITS; ++j) {
            pos[j] = int(std::find(ps.window.begin(), ps.window.end(), op.qubits[j]) - ps.window.begin());
            gt |= 1u << pos[j];
          }
          std::vector<CplxD> in(32), outv(32);
          for (uint32_t e = 0; e < t.size(); ++e) {
            if (e & gt) continue;  // one column: the gate bits zero
            for (uint32_t r = 0; r < 32; ++r) {
              uint32_t ee = e;
              for (int j = 0; j < GROUP_QUBITS; ++j) ee |= ((r >> j) & 1) << pos[j];
              in[r] = t[ee];
            }
            for (uint32_t r = 0; r < 32; ++r) {
              CplxD acc{0, 0};
              for (uint32_t k = 0; k < 32; ++k) {
                CplxD m = mul(op.u[r * 32 + k], in[k]);
                acc.re += m.re;
                acc.im += m.im;
              }
              outv[r] = acc;
            }
            for (uint32_t r = 0; r < 32; ++r) {
              uint32_t ee = e;
              for (int j = 0; j < GROUP_QUBITS; ++j) ee |= ((r >> j) & 1) << pos[j];
              t[ee] = outv[r];
            }
          }
        }
        for (uint32_t e = 0; e < t.size(); ++e) a[gidx(e)] = t[e];
      }
    }
  }
}

}  // namespace fused
}  // namespace ncsim
