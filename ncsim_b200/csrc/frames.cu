// Pauli-frame sampling of noisy Clifford circuits on the GPU (the reference's
// FrameSampler, src/frame.rs:34-300).
//
// The frames of all shots are bit-sliced: qubit q's x (and z) bits of 64
// shots are one word.  A shot-word never interacts with another, so a CTA
// owns W consecutive shot-words (lane = word) for the whole circuit and keeps
// their 2n frame columns in shared memory (global memory when 16 n W bytes do
// not fit); its S = 256 / W slots apply the operations of one dependency
// layer of the circuit in parallel (operations of a layer touch disjoint
// qubits), with one barrier per layer.  No CTA waits for another.
//
// The random masks (ChaCha12 words of each batch's StdRng at positions the
// host scan computed) are expanded by their own kernel, 8 words a thread; the
// noise hits, whose geometric skips need the host's log() to match the
// reference draw for draw, arrive from the host scan as per-op lists.
#include <algorithm>
#include <atomic>
#include <thread>

#include "engine.cuh"
#include "frames_plan.hpp"

using namespace ncsim;
using namespace ncsim::frames;

namespace {

constexpr int FRAME_THREADS = 256;
constexpr size_t FRAME_SMEM_CAP = 200 * 1024;

// ---------------------------------------------------------------------------
// ChaCha12 block (RFC 8439 quarter round; rand_chacha's StdRng: 12 rounds,
// 64-bit block counter in words 12-13, stream 0 in words 14-15)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t rotl(uint32_t v, int s) { return __funnelshift_l(v, v, s); }

__device__ __forceinline__ void chacha12_block(const uint32_t* __restrict__ key, uint64_t ctr, uint32_t out[16]) {
  uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                    key[4],      key[5],      key[6],      key[7],      uint32_t(ctr), uint32_t(ctr >> 32), 0u, 0u};
  uint32_t in[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) in[i] = s[i];
#define NCSIM_DQR(a, b, c, d)        \
  s[a] += s[b];                      \
  s[d] = rotl(s[d] ^ s[a], 16);      \
  s[c] += s[d];                      \
  s[b] = rotl(s[b] ^ s[c], 12);      \
  s[a] += s[b];                      \
  s[d] = rotl(s[d] ^ s[a], 8);       \
  s[c] += s[d];                      \
  s[b] = rotl(s[b] ^ s[c], 7)
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    NCSIM_DQR(0, 4, 8, 12);
    NCSIM_DQR(1, 5, 9, 13);
    NCSIM_DQR(2, 6, 10, 14);
    NCSIM_DQR(3, 7, 11, 15);
    NCSIM_DQR(0, 5, 10, 15);
    NCSIM_DQR(1, 6, 11, 12);
    NCSIM_DQR(2, 7, 8, 13);
    NCSIM_DQR(3, 4, 9, 14);
  }
#undef NCSIM_DQR
#pragma unroll
  for (int i = 0; i < 16; ++i) out[i] = s[i] + in[i];
}

// the valid-shot bits of shot-word g (only the last batch can be partial)
__device__ __forceinline__ uint64_t valid_bits(uint64_t g, uint64_t shots) {
  const uint64_t first = g * 64;
  if (first >= shots) return 0;
  const uint64_t left = shots - first;
  return left >= 64 ? ~uint64_t(0) : ((uint64_t(1) << left) - 1);
}

// masks[j * G + g]: random_mask j of the batch holding word g (frame.rs:107-111),
// 8 words per thread
__global__ void __launch_bounds__(256) k_frame_masks(const uint32_t* __restrict__ keys, const uint64_t* __restrict__ pos,
                                                     uint32_t J, uint64_t G, uint64_t shots,
                                                     uint64_t* __restrict__ masks) {
  const uint64_t G8 = (G + 7) / 8;
  const uint64_t items = uint64_t(J) * G8;
  for (uint64_t it = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; it < items;
       it += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t j = uint32_t(it / G8);
    const uint64_t g0 = (it % G8) * 8;
    const uint64_t b = g0 / BATCH_WORDS;
    const uint64_t P = pos[b * J + j] + 2 * (g0 % BATCH_WORDS);  // even: draws are u64 pairs
    const uint32_t* key = keys + 8 * b;
    uint32_t blk[32];
    chacha12_block(key, P / 16, blk);
    const uint32_t off = uint32_t(P % 16);
    if (off) chacha12_block(key, P / 16 + 1, blk + 16);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint64_t g = g0 + u;
      if (g >= G) break;
      const uint32_t w = off + 2 * u;
      const uint64_t v = uint64_t(blk[w]) | (uint64_t(blk[w + 1]) << 32);
      masks[uint64_t(j) * G + g] = v & valid_bits(g, shots);
    }
  }
}

struct RunParams {
  const FrameOp* ops;
  const uint32_t* layer_off;
  uint32_t nlayers;
  const uint32_t* pool;
  const uint64_t* masks;
  uint64_t* recs;
  uint64_t G, shots;
  uint32_t n, W, NI;
  const uint32_t* ev_off;   // per batch: NI + 1 offsets
  const uint32_t* ev_base;  // per batch: first event
  const uint32_t* events;
  uint64_t* gtab;           // per-CTA tables when they do not fit in shared memory
};

template <bool SHARED>
__global__ void __launch_bounds__(FRAME_THREADS) k_frame_run(const RunParams P) {
  extern __shared__ __align__(16) uint64_t frame_smem[];
  const uint32_t W = P.W, S = blockDim.x / W;
  const uint32_t lane = threadIdx.x % W, slot = threadIdx.x / W;
  uint64_t* tab = SHARED ? frame_smem : P.gtab + uint64_t(blockIdx.x) * 2 * P.n * W;
  const uint64_t g = uint64_t(blockIdx.x) * W + lane;
  const bool active = g < P.G;
  const uint64_t valid = active ? valid_bits(g, P.shots) : 0;
  const uint32_t b = uint32_t(g / BATCH_WORDS), wb = uint32_t(g % BATCH_WORDS);
#define XQ(q) tab[(2 * uint64_t(q)) * W + lane]
#define ZQ(q) tab[(2 * uint64_t(q) + 1) * W + lane]
  // every qubit's frame starts as Z with a random mask (frame.rs:112-115)
  for (uint32_t q = slot; q < P.n; q += S) {
    XQ(q) = 0;
    ZQ(q) = active ? P.masks[uint64_t(q) * P.G + g] : 0;
  }
  __syncthreads();
  for (uint32_t L = 0; L < P.nlayers; ++L) {
    const uint32_t hi = P.layer_off[L + 1];
    for (uint32_t o = P.layer_off[L] + slot; o < hi; o += S) {
      const FrameOp op = P.ops[o];
      const uint32_t kind = op.kind & 0xff;
      switch (kind) {
        case FOP_H: {
          const uint64_t x = XQ(op.a);
          XQ(op.a) = ZQ(op.a);
          ZQ(op.a) = x;
          break;
        }
        case FOP_S: ZQ(op.a) ^= XQ(op.a); break;
        case FOP_SQRTX: XQ(op.a) ^= ZQ(op.a); break;
        case FOP_CX: {
          const uint64_t xa = XQ(op.a), zb = ZQ(op.b);
          XQ(op.b) ^= xa;
          ZQ(op.a) ^= zb;
          break;
        }
        case FOP_CZ: {
          const uint64_t xa = XQ(op.a), xb = XQ(op.b);
          ZQ(op.a) ^= xb;
          ZQ(op.b) ^= xa;
          break;
        }
        case FOP_SWAP: {
          const uint64_t xa = XQ(op.a), za = ZQ(op.a);
          XQ(op.a) = XQ(op.b);
          ZQ(op.a) = ZQ(op.b);
          XQ(op.b) = xa;
          ZQ(op.b) = za;
          break;
        }
        case FOP_LINEAR: {
          const uint32_t k = (op.kind >> 8) & 0xff;
          const uint32_t* qs = P.pool + op.off;
          const uint32_t* rows = qs + k;
          uint64_t in[2 * MAX_LINEAR_K], out[2 * MAX_LINEAR_K];
          for (uint32_t j = 0; j < k; ++j) {
            in[2 * j] = XQ(qs[j]);
            in[2 * j + 1] = ZQ(qs[j]);
          }
          for (uint32_t i = 0; i < 2 * k; ++i) {
            const uint64_t row = uint64_t(rows[2 * i]) | (uint64_t(rows[2 * i + 1]) << 32);
            uint64_t acc = 0;
            for (uint32_t t = 0; t < 2 * k; ++t)
              if ((row >> t) & 1) acc ^= in[t];
            out[i] = acc;
          }
          for (uint32_t j = 0; j < k; ++j) {
            XQ(qs[j]) = out[2 * j];
            ZQ(qs[j]) = out[2 * j + 1];
          }
          break;
        }
        case FOP_MEASURE: {
          // record = reference ^ [frame anticommutes with P], then the frame
          // is randomised by P (frame.rs:120-133)
          const uint32_t cnt = (op.kind >> 8) & 0x7fffff;
          const uint32_t* sites = P.pool + op.off;
          uint64_t rec = 0;
          for (uint32_t t = 0; t < cnt; ++t) {
            const uint32_t q = sites[t] & 0xffffff, l = sites[t] >> 24;
            if (l & 1) rec ^= ZQ(q);
            if (l & 2) rec ^= XQ(q);
          }
          if (op.kind >> 31) rec = ~rec;
          rec &= valid;
          if (active) P.recs[uint64_t(op.a) * P.G + g] = rec;
          const uint64_t r = active ? P.masks[uint64_t(op.b) * P.G + g] : 0;
          for (uint32_t t = 0; t < cnt; ++t) {
            const uint32_t q = sites[t] & 0xffffff, l = sites[t] >> 24;
            if (l & 1) XQ(q) ^= r;
            if (l & 2) ZQ(q) ^= r;
          }
          break;
        }
        case FOP_RESET:
          XQ(op.a) = 0;
          ZQ(op.a) = active ? P.masks[uint64_t(op.b) * P.G + g] : 0;
          break;
        case FOP_NOISE: {
          if (!active) break;
          const uint32_t k = (op.kind >> 8) & 0xff;
          const uint32_t* qs = P.pool + op.off;
          const uint32_t* eo = P.ev_off + uint64_t(b) * (P.NI + 1);
          const uint32_t base = P.ev_base[b];
          const uint32_t end = base + eo[op.a + 1];
          for (uint32_t e = base + eo[op.a]; e < end; ++e) {
            const uint32_t ev = P.events[e];
            const uint32_t s = ev & 0xffff;
            if ((s >> 6) < wb) continue;
            if ((s >> 6) > wb) break;  // hits are in shot order
            const uint64_t bit = uint64_t(1) << (s & 63);
            const uint32_t ex = (ev >> 16) & 0xf, ez = (ev >> 20) & 0xf;
            for (uint32_t j = 0; j < k; ++j) {
              if ((ex >> j) & 1) XQ(qs[j]) ^= bit;
              if ((ez >> j) & 1) ZQ(qs[j]) ^= bit;
            }
          }
          break;
        }
        default: break;
      }
    }
    __syncthreads();
  }
#undef XQ
#undef ZQ
}

// out[d * G + g] = flip_d ^ parity of the records listed for d (frame.rs:155-205, 296-307)
__global__ void __launch_bounds__(256) k_frame_parity(const uint64_t* __restrict__ recs, uint64_t G, uint64_t shots,
                                                      const uint32_t* __restrict__ off, const uint32_t* __restrict__ idx,
                                                      const uint8_t* __restrict__ flip, uint32_t count,
                                                      uint64_t* __restrict__ out) {
  const uint64_t items = uint64_t(count) * G;
  for (uint64_t it = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; it < items;
       it += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t d = uint32_t(it / G);
    const uint64_t g = it % G;
    uint64_t acc = 0;
    for (uint32_t t = off[d]; t < off[d + 1]; ++t) acc ^= recs[uint64_t(idx[t]) * G + g];
    if (flip[d]) acc = ~acc;
    out[it] = acc & valid_bits(g, shots);
  }
}

// per-shot records (bit k of shot s) from the packed ones (frame.rs:91-102)
__global__ void __launch_bounds__(256) k_frame_transpose(const uint64_t* __restrict__ recs, uint64_t G, uint64_t shots,
                                                         uint64_t m, uint64_t* __restrict__ out) {
  const uint64_t MW = (m + 63) / 64;
  const uint64_t items = shots * MW;
  for (uint64_t it = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; it < items;
       it += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t kw = it / shots, s = it % shots;
    uint64_t v = 0;
    for (uint32_t t = 0; t < 64; ++t) {
      const uint64_t k = kw * 64 + t;
      if (k >= m) break;
      v |= ((recs[k * G + s / 64] >> (s & 63)) & 1) << t;
    }
    out[s * MW + kw] = v;
  }
}

unsigned grid_of(uint64_t items, unsigned threads) {
  const uint64_t want = (items + threads - 1) / threads;
  return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(sm_count()) * 16)));
}

template <class F>
void each_batch(size_t count, F&& f) {
  std::atomic<size_t> next{0};
  std::vector<std::string> errs(count);
  auto work = [&] {
    for (size_t i; (i = next.fetch_add(1)) < count;) {
      try {
        f(i);
      } catch (const std::exception& e) {
        errs[i] = e.what();
      }
    }
  };
  const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  const unsigned nth = unsigned(std::min<size_t>(hw, count));
  std::vector<std::thread> th;
  for (unsigned k = 1; k < nth; ++k) th.emplace_back(work);
  work();
  for (auto& x : th) x.join();
  for (auto& e : errs)
    if (!e.empty()) throw Error(NCSIM_ERR_INVALID, e);
}

// device buffer that only grows
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  void ensure(size_t n) {
    if (n <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    NCSIM_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    cap = n;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};
template <class T>
struct HostBuf {
  T* p = nullptr;
  size_t cap = 0;
  void ensure(size_t n) {
    if (n <= cap) return;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    NCSIM_CUDA(cudaMallocHost(&p, std::max<size_t>(n, 1) * sizeof(T)));
    cap = n;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace

struct ncsim_frames {
  Program prog;
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_kernel_ms = 0.f;
  uint32_t W = 0;
  bool shared = true;
  // the program on the device
  DevBuf<FrameOp> d_ops;
  DevBuf<uint32_t> d_layers, d_pool;
  DevBuf<uint32_t> d_det_off, d_det_idx, d_obs_off, d_obs_idx;
  DevBuf<uint8_t> d_det_flip, d_obs_flip;
  // per call
  DevBuf<uint32_t> d_keys, d_ev_off, d_ev_base, d_events;
  DevBuf<uint64_t> d_pos, d_masks, d_recs, d_gtab, d_out;
  HostBuf<uint32_t> h_keys, h_ev_off, h_ev_base, h_events;
  HostBuf<uint64_t> h_pos;
  std::vector<BatchScan> scans;

  ~ncsim_frames() {
    if (device >= 0) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(device);
      if (stream) cudaStreamSynchronize(stream);
      d_ops.release();
      d_layers.release();
      d_pool.release();
      d_det_off.release();
      d_det_idx.release();
      d_obs_off.release();
      d_obs_idx.release();
      d_det_flip.release();
      d_obs_flip.release();
      d_keys.release();
      d_ev_off.release();
      d_ev_base.release();
      d_events.release();
      d_pos.release();
      d_masks.release();
      d_recs.release();
      d_gtab.release();
      d_out.release();
      h_keys.release();
      h_ev_off.release();
      h_ev_base.release();
      h_events.release();
      h_pos.release();
      if (ev0) cudaEventDestroy(ev0);
      if (ev1) cudaEventDestroy(ev1);
      if (stream) cudaStreamDestroy(stream);
      cudaSetDevice(cur);
    }
  }
};

namespace {

template <class T>
void upload(DevBuf<T>& d, const std::vector<T>& v, cudaStream_t st) {
  d.ensure(v.size());
  if (!v.empty()) NCSIM_CUDA(cudaMemcpyAsync(d.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

void index_lists(const std::vector<std::vector<uint64_t>>& lists, std::vector<uint32_t>& off, std::vector<uint32_t>& idx) {
  off.assign(1, 0);
  idx.clear();
  for (auto& l : lists) {
    for (uint64_t k : l) idx.push_back(uint32_t(k));
    off.push_back(uint32_t(idx.size()));
  }
}

// the device program, on the device that is current at first use
void ensure_device(ncsim_frames* f) {
  int dev = 0;
  NCSIM_CUDA(cudaGetDevice(&dev));
  if (f->device == dev) return;
  if (f->device >= 0) throw Error(NCSIM_ERR_DEVICE, "a frame sampler stays on the device it first ran on");
  f->device = dev;
  NCSIM_CUDA(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking));
  NCSIM_CUDA(cudaEventCreate(&f->ev0));
  NCSIM_CUDA(cudaEventCreate(&f->ev1));
  const Program& p = f->prog;
  upload(f->d_ops, p.ops, f->stream);
  upload(f->d_layers, p.layer_off, f->stream);
  upload(f->d_pool, p.pool, f->stream);
  std::vector<uint32_t> off, idx;
  index_lists(p.detectors, off, idx);
  upload(f->d_det_off, off, f->stream);
  upload(f->d_det_idx, idx, f->stream);
  upload(f->d_det_flip, p.det_flip, f->stream);
  index_lists(p.observables, off, idx);
  upload(f->d_obs_off, off, f->stream);
  upload(f->d_obs_idx, idx, f->stream);
  upload(f->d_obs_flip, p.obs_flip, f->stream);
  NCSIM_CUDA(cudaStreamSynchronize(f->stream));
}

// words per CTA: shared-memory tables when 16 n W bytes fit, as many CTAs as
// the SMs can hold at once when the shots allow it, at least a 32-byte sector
// of words where there are enough of them
void choose_shape(ncsim_frames* f, uint64_t G) {
  const uint64_t n = std::max<uint32_t>(f->prog.n, 1);
  uint32_t W = 32;
  while (W > 1 && 16 * n * W > FRAME_SMEM_CAP) W /= 2;
  f->shared = 16 * n * W <= FRAME_SMEM_CAP;
  if (!f->shared) W = 32;
  const uint64_t want_ctas = uint64_t(sm_count()) * 2;
  while (W > 4 && (G + W - 1) / W < want_ctas) W /= 2;
  f->W = W;
}

// scan, upload, expand the masks and run the frames: records in d_recs ([k][G])
void run_frames(ncsim_frames* f, uint64_t shots, const uint64_t* seeds, uint64_t nseeds) {
  const Program& p = f->prog;
  const uint64_t nb = (shots + BATCH - 1) / BATCH;
  if (nseeds != nb)
    throw Error(NCSIM_ERR_INVALID, std::to_string(shots) + " shots take " + std::to_string(nb) + " batch seeds, " +
                                       std::to_string(nseeds) + " given");
  if (shots == 0) return;
  if (!seeds) throw Error(NCSIM_ERR_INVALID, "null seeds");
  ensure_device(f);
  const uint64_t G = (shots + 63) / 64;
  const uint32_t J = p.num_masks;
  const uint32_t NI = uint32_t(p.noise.size());
  // the host scan of every batch's stream, batches in parallel
  f->scans.resize(nb);
  each_batch(nb, [&](size_t b) {
    const uint32_t size = uint32_t(std::min<uint64_t>(BATCH, shots - b * BATCH));
    scan_batch(p, seeds[b], size, f->scans[b]);
  });
  uint64_t nev = 0;
  for (auto& s : f->scans) nev += s.events.size();
  if (nev >= (uint64_t(1) << 32)) throw Error(NCSIM_ERR_UNSUPPORTED, "more than 2^32 noise hits in one call");
  f->h_keys.ensure(nb * 8);
  f->h_pos.ensure(nb * J);
  f->h_ev_off.ensure(nb * (NI + 1));
  f->h_ev_base.ensure(nb);
  f->h_events.ensure(nev);
  uint64_t base = 0;
  for (uint64_t b = 0; b < nb; ++b) {
    key_of_seed(seeds[b], f->h_keys.p + 8 * b);
    std::copy(f->scans[b].mask_pos.begin(), f->scans[b].mask_pos.end(), f->h_pos.p + b * J);
    std::copy(f->scans[b].ev_off.begin(), f->scans[b].ev_off.end(), f->h_ev_off.p + b * (NI + 1));
    f->h_ev_base.p[b] = uint32_t(base);
    std::copy(f->scans[b].events.begin(), f->scans[b].events.end(), f->h_events.p + base);
    base += f->scans[b].events.size();
  }
  cudaStream_t st = f->stream;
  f->d_keys.ensure(nb * 8);
  f->d_pos.ensure(nb * J);
  f->d_ev_off.ensure(nb * (NI + 1));
  f->d_ev_base.ensure(nb);
  f->d_events.ensure(nev);
  f->d_masks.ensure(uint64_t(J) * G);
  f->d_recs.ensure(std::max<uint64_t>(p.num_measurements, 1) * G);
  NCSIM_CUDA(cudaMemcpyAsync(f->d_keys.p, f->h_keys.p, nb * 8 * 4, cudaMemcpyHostToDevice, st));
  NCSIM_CUDA(cudaMemcpyAsync(f->d_pos.p, f->h_pos.p, nb * J * 8, cudaMemcpyHostToDevice, st));
  NCSIM_CUDA(cudaMemcpyAsync(f->d_ev_off.p, f->h_ev_off.p, nb * (NI + 1) * 4, cudaMemcpyHostToDevice, st));
  NCSIM_CUDA(cudaMemcpyAsync(f->d_ev_base.p, f->h_ev_base.p, nb * 4, cudaMemcpyHostToDevice, st));
  if (nev) NCSIM_CUDA(cudaMemcpyAsync(f->d_events.p, f->h_events.p, nev * 4, cudaMemcpyHostToDevice, st));
  choose_shape(f, G);
  const uint32_t W = f->W;
  const uint64_t ctas = (G + W - 1) / W;
  if (ctas > 0x7fffffffu) throw Error(NCSIM_ERR_UNSUPPORTED, "too many shots for one call");
  RunParams rp;
  rp.ops = f->d_ops.p;
  rp.layer_off = f->d_layers.p;
  rp.nlayers = uint32_t(p.layer_off.size() - 1);
  rp.pool = f->d_pool.p;
  rp.masks = f->d_masks.p;
  rp.recs = f->d_recs.p;
  rp.G = G;
  rp.shots = shots;
  rp.n = p.n;
  rp.W = W;
  rp.NI = NI;
  rp.ev_off = f->d_ev_off.p;
  rp.ev_base = f->d_ev_base.p;
  rp.events = f->d_events.p;
  rp.gtab = nullptr;
  NCSIM_CUDA(cudaEventRecord(f->ev0, st));
  if (J) {
    k_frame_masks<<<grid_of(uint64_t(J) * ((G + 7) / 8), 256), 256, 0, st>>>(f->d_keys.p, f->d_pos.p, J, G, shots,
                                                                             f->d_masks.p);
    NCSIM_LAUNCHED("k_frame_masks");
  }
  const unsigned threads = (FRAME_THREADS / W) * W;
  if (f->shared) {
    const size_t smem = size_t(16) * p.n * W;
    NCSIM_CUDA(cudaFuncSetAttribute(k_frame_run<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k_frame_run<true><<<unsigned(ctas), threads, smem, st>>>(rp);
  } else {
    f->d_gtab.ensure(ctas * 2 * uint64_t(p.n) * W);
    rp.gtab = f->d_gtab.p;
    k_frame_run<false><<<unsigned(ctas), threads, 0, st>>>(rp);
  }
  NCSIM_LAUNCHED("k_frame_run");
  NCSIM_CUDA(cudaEventRecord(f->ev1, st));
}

void finish(ncsim_frames* f) {
  NCSIM_CUDA(cudaStreamSynchronize(f->stream));
  NCSIM_CUDA(cudaEventElapsedTime(&f->last_kernel_ms, f->ev0, f->ev1));
}

std::vector<uint64_t> seeds_from(ncsim_rng* rng, uint64_t shots) {
  if (!rng) throw Error(NCSIM_ERR_INVALID, "null generator");
  std::vector<uint64_t> s((shots + BATCH - 1) / BATCH);
  for (auto& v : s) v = rng->u64();  // one draw per batch, in order (frame.rs:72-74)
  return s;
}

void check_cap(uint64_t need, uint64_t cap, const char* what) {
  if (need > cap) throw Error(NCSIM_ERR_INVALID, std::string(what) + ": needs " + std::to_string(need) + " words, " +
                                                     std::to_string(cap) + " given");
}

void packed_seeds(ncsim_frames* f, uint64_t shots, const uint64_t* seeds, uint64_t nseeds, uint64_t* out, uint64_t cap,
                  bool device_out) {
  const uint64_t G = (shots + 63) / 64, m = f->prog.num_measurements;
  check_cap(m * G, cap, "sample_packed");
  if (m * G && !out) throw Error(NCSIM_ERR_INVALID, "null output");
  run_frames(f, shots, seeds, nseeds);
  if (shots && m)
    NCSIM_CUDA(cudaMemcpyAsync(out, f->d_recs.p, m * G * 8, device_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                               f->stream));
  if (shots) finish(f);
}

void detectors_seeds(ncsim_frames* f, uint64_t shots, const uint64_t* seeds, uint64_t nseeds, uint64_t* det,
                     uint64_t det_cap, uint64_t* obs, uint64_t obs_cap) {
  const Program& p = f->prog;
  const uint64_t G = (shots + 63) / 64;
  const uint64_t nd = p.detectors.size(), no = p.observables.size();
  check_cap(nd * G, det_cap, "detectors");
  check_cap(no * G, obs_cap, "observables");
  if ((nd * G && !det) || (no * G && !obs)) throw Error(NCSIM_ERR_INVALID, "null output");
  run_frames(f, shots, seeds, nseeds);
  if (!shots) return;
  f->d_out.ensure(std::max<uint64_t>(nd + no, 1) * G);
  if (nd) {
    k_frame_parity<<<grid_of(nd * G, 256), 256, 0, f->stream>>>(f->d_recs.p, G, shots, f->d_det_off.p, f->d_det_idx.p,
                                                                f->d_det_flip.p, uint32_t(nd), f->d_out.p);
    NCSIM_LAUNCHED("k_frame_parity");
    NCSIM_CUDA(cudaMemcpyAsync(det, f->d_out.p, nd * G * 8, cudaMemcpyDeviceToHost, f->stream));
  }
  if (no) {
    k_frame_parity<<<grid_of(no * G, 256), 256, 0, f->stream>>>(f->d_recs.p, G, shots, f->d_obs_off.p, f->d_obs_idx.p,
                                                                f->d_obs_flip.p, uint32_t(no), f->d_out.p + nd * G);
    NCSIM_LAUNCHED("k_frame_parity");
    NCSIM_CUDA(cudaMemcpyAsync(obs, f->d_out.p + nd * G, no * G * 8, cudaMemcpyDeviceToHost, f->stream));
  }
  finish(f);
}

void shots_seeds(ncsim_frames* f, uint64_t shots, const uint64_t* seeds, uint64_t nseeds, uint64_t* out, uint64_t cap) {
  const uint64_t m = f->prog.num_measurements, MW = (m + 63) / 64, G = (shots + 63) / 64;
  check_cap(shots * MW, cap, "sample");
  if (shots * MW && !out) throw Error(NCSIM_ERR_INVALID, "null output");
  run_frames(f, shots, seeds, nseeds);
  if (!shots || !m) return;
  f->d_out.ensure(shots * MW);
  k_frame_transpose<<<grid_of(shots * MW, 256), 256, 0, f->stream>>>(f->d_recs.p, G, shots, m, f->d_out.p);
  NCSIM_LAUNCHED("k_frame_transpose");
  NCSIM_CUDA(cudaMemcpyAsync(out, f->d_out.p, shots * MW * 8, cudaMemcpyDeviceToHost, f->stream));
  finish(f);
}

}  // namespace

extern "C" {

ncsim_status ncsim_frames_new(const ncsim_circuit* c, uint64_t reference_seed, ncsim_frames** out) {
  return guarded([&] {
    if (!c || !out) throw Error(NCSIM_ERR_INVALID, "null argument");
    *out = nullptr;
    // the Clifford check comes first, as in FrameSampler::new
    for (const auto& op : c->ops) {
      CliffordAction a;
      if (op.kind == OpKind::Gate && !clifford_action(op.gate, a))
        throw Error(NCSIM_ERR_UNSUPPORTED, "FrameSampler: non-Clifford gate " + op.gate.text());
    }
    const std::vector<uint8_t> ref = reference_record(*c, reference_seed);
    auto* f = new ncsim_frames();
    try {
      f->prog = compile(*c, ref);
    } catch (...) {
      delete f;
      throw;
    }
    *out = f;
  });
}

ncsim_status ncsim_frames_with_reference(const ncsim_circuit* c, const uint8_t* reference, uint64_t m,
                                         ncsim_frames** out) {
  return guarded([&] {
    if (!c || !out || (m && !reference)) throw Error(NCSIM_ERR_INVALID, "null argument");
    *out = nullptr;
    std::vector<uint8_t> ref(reference, reference + m);
    for (auto& r : ref) r = r ? 1 : 0;
    auto* f = new ncsim_frames();
    try {
      f->prog = compile(*c, ref);
    } catch (...) {
      delete f;
      throw;
    }
    *out = f;
  });
}

ncsim_status ncsim_frames_free(ncsim_frames* f) {
  return guarded([&] { delete f; });
}

ncsim_status ncsim_frames_info(const ncsim_frames* f, uint32_t* num_qubits, uint64_t* num_measurements,
                               uint64_t* num_detectors, uint64_t* num_observables, uint64_t* num_layers) {
  return guarded([&] {
    if (!f) throw Error(NCSIM_ERR_INVALID, "null sampler");
    if (num_qubits) *num_qubits = f->prog.n;
    if (num_measurements) *num_measurements = f->prog.num_measurements;
    if (num_detectors) *num_detectors = f->prog.detectors.size();
    if (num_observables) *num_observables = f->prog.observables.size();
    if (num_layers) *num_layers = f->prog.layer_off.size() - 1;
  });
}

ncsim_status ncsim_frames_reference(const ncsim_frames* f, uint8_t* out, uint64_t cap) {
  return guarded([&] {
    if (!f) throw Error(NCSIM_ERR_INVALID, "null sampler");
    const auto& r = f->prog.reference;
    if (cap < r.size()) throw Error(NCSIM_ERR_INVALID, "reference: buffer too small");
    if (!r.empty() && !out) throw Error(NCSIM_ERR_INVALID, "null output");
    std::copy(r.begin(), r.end(), out);
  });
}

ncsim_status ncsim_frames_sample_packed(ncsim_frames* f, uint64_t shots, ncsim_rng* rng, uint64_t* out, uint64_t cap) {
  return guarded([&] {
    if (!f) throw Error(NCSIM_ERR_INVALID, "null sampler");
    const auto seeds = seeds_from(rng, shots);
    packed_seeds(f, shots, seeds.data(), seeds.size(), out, cap, false);
  });
}

ncsim_status ncsim_frames_sample_packed_seeds(ncsim_frames* f, uint64_t shots, const uint64_t* seeds, uint64_t nseeds,
                                              uint64_t* out, uint64_t cap) {
  return guarded([&] {
    if (!f) throw Error(NCSIM_ERR_INVALID, "null sampler");
    packed_seeds(f, shots, seeds, nseeds, out, cap, false);
  });
}

ncsim_status ncsim_frames_sample_packed_device(ncsim_frames* f, uint64_t shots, const uint64_t* seeds, uint64_t nseeds,
                                               uint64_t* d_out, uint64_t cap) {
  return guarded([&] {
    if (!f) throw Error(NCSIM_ERR_INVALID, "null sampler");
    packed_seeds(f, shots, seeds, nseeds, d_out, cap, true);
  });
}

ncsim_status ncsim_frames_sample(ncsim_frames* f, uint64_t shots, ncsim_rng* rng, uint64_t* out, uint64_t cap) {
  return guarded([&] {
    if (!f) throw Error(NCSIM_ERR_INVALID, "null sampler");
    const auto seeds = seeds_from(rng, shots);
    shots_seeds(f, shots, seeds.data(), seeds.size(), out, cap);
  });
}

ncsim_status ncsim_frames_sample_detectors(ncsim_frames* f, uint64_t shots, ncsim_rng* rng, uint64_t* det,
                                           uint64_t det_cap, uint64_t* obs, uint64_t obs_cap) {
  return guarded([&] {
    if (!f) throw Error(NCSIM_ERR_INVALID, "null sampler");
    const auto seeds = seeds_from(rng, shots);
    detectors_seeds(f, shots, seeds.data(), seeds.size(), det, det_cap, obs, obs_cap);
  });
}

ncsim_status ncsim_frames_sample_detectors_seeds(ncsim_frames* f, uint64_t shots, const uint64_t* seeds,
                                                 uint64_t nseeds, uint64_t* det, uint64_t det_cap, uint64_t* obs,
                                                 uint64_t obs_cap) {
  return guarded([&] {
    if (!f) throw Error(NCSIM_ERR_INVALID, "null sampler");
    detectors_seeds(f, shots, seeds, nseeds, det, det_cap, obs, obs_cap);
  });
}

ncsim_status ncsim_frames_last_kernel_ms(const ncsim_frames* f, double* ms) {
  return guarded([&] {
    if (!f || !ms) throw Error(NCSIM_ERR_INVALID, "null argument");
    *ms = double(f->last_kernel_ms);
  });
}

}  // extern "C"
