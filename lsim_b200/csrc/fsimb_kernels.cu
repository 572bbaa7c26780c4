// B200 (sm_100a) kernels of the stuck-at fault simulator.
//
//   k_good_level   good machine, one launch per level, one thread per
//                  (element, word); warps cover the 32 words of a tile so every
//                  fanin read is one coalesced 256-byte segment.
//   k_sweep<M>     persistent: each CTA pulls (sweep, M-word subtile) items from
//                  a device work counter and re-simulates the levels above the
//                  injection point with all live values in shared memory
//                  (slots assigned on the host by interval allocation).  Writes
//                  the OR over POs of (faulty ^ good) per word.
//   k_ffr          one warp per FFR root, lanes = the 32 words of a tile:
//                  backward critical-path tracing inside the FFR and the
//                  per-fault detection word, count and first pattern.
//   k_exact        the same epilogue for faults simulated by an exact sweep.
//   k_drop         fault dropping: warp-aggregated stream compaction of the
//                  roots / sweeps that still carry undetected faults.
//
// Word semantics follow fsim/simulation.cpp: gates act on whole 64-bit words
// (fsim/simulation.cpp:979-1124), the last round keeps its high bits until
// the PO comparison masks them (fsim/simulation.cpp:94-102, 174-178), and a
// detecting bit b of round rd with `bits` valid bits is pattern
// rd*64 + bits-1-b.
#include "fsimb_kernels.cuh"

namespace fsimb {

namespace {

// Gate families: AND/OR/NAND/NOR/INV/CLKBUF/PO are io ^ AND(in ^ ii);
// XOR/XNOR are io ^ XOR(in).  Bit t of each mask is the property of type t.
constexpr uint32_t kIiMask = (1u << G_OR) | (1u << G_NOR);
constexpr uint32_t kIoMask = (1u << G_INV) | (1u << G_OR) | (1u << G_NAND) | (1u << G_XNOR);
constexpr uint32_t kXfMask = (1u << G_XOR) | (1u << G_XNOR);

__device__ __forceinline__ uint64_t bmask(uint32_t bit) { return 0ull - (uint64_t)bit; }

// Evaluates one word.  in[k] for k >= nf is ignored.
__device__ __forceinline__ uint64_t eval_word(uint32_t t, uint32_t nf, uint64_t a, uint64_t b,
                                              uint64_t c, uint64_t d) {
  if (t == G_MUX) {
    // (s & b) | (a & !s) with a logical not (fsim/simulation.cpp:1056)
    return (c & b) | (a & (uint64_t)(c == 0));
  }
  const uint64_t ii = bmask((kIiMask >> t) & 1u);
  const uint64_t io = bmask((kIoMask >> t) & 1u);
  const bool xf = (kXfMask >> t) & 1u;
  const uint64_t fill_ao = ~ii;
  if (nf < 2) b = xf ? 0ull : fill_ao;
  if (nf < 3) c = xf ? 0ull : fill_ao;
  if (nf < 4) d = xf ? 0ull : fill_ao;
  const uint64_t ao = (a ^ ii) & (b ^ ii) & (c ^ ii) & (d ^ ii);
  const uint64_t xo = a ^ b ^ c ^ d;
  return (xf ? xo : ao) ^ io;
}

__device__ __forceinline__ uint32_t round_bits(uint64_t P, uint32_t W, uint32_t w) {
  if (w >= W) return 0;
  return (P / (64ull * (w + 1))) ? 64u : (uint32_t)(P % 64);
}

__device__ __forceinline__ uint64_t bits_mask(uint32_t bits) {
  return bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
}

// ---------------------------------------------------------------- good
__global__ void k_good_level(GoodArgs a) {
  const uint64_t n = (uint64_t)(a.hi - a.lo) * a.W_pad;
  for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t w = (uint32_t)(idx % a.W_pad);
    const uint32_t e = a.lo + (uint32_t)(idx / a.W_pad);
    const uint32_t tile = w >> 5, lane = w & 31u;
    const uint64_t base = (uint64_t)tile * a.N;
    const uint8_t t = a.type[e];
    uint64_t v;
    if (t == G_PI) {
      v = (w < a.W) ? a.pwords[(uint64_t)w * a.n_pi + e] : 0ull;
    } else {
      const uint32_t f0 = a.fi_off[e];
      uint32_t nf = a.fi_off[e + 1] - f0;
      if (t == G_INV || t == G_CLKBUF || t == G_PO) nf = 1;
      uint64_t in[4] = {0, 0, 0, 0};
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if ((uint32_t)k < nf) in[k] = a.good[(base + a.fi_idx[f0 + k]) * 32 + lane];
      v = eval_word(t, nf, in[0], in[1], in[2], in[3]);
    }
    a.good[(base + e) * 32 + lane] = v;
  }
}

// ---------------------------------------------------------------- sweep
template <int M>
__device__ __forceinline__ void ld_words(const uint64_t* p, uint64_t (&v)[M]) {
  if constexpr (M == 1) {
    v[0] = p[0];
  } else {
#pragma unroll
    for (int i = 0; i < M / 2; ++i) {
      ulonglong2 q = reinterpret_cast<const ulonglong2*>(p)[i];
      v[2 * i] = q.x;
      v[2 * i + 1] = q.y;
    }
  }
}

template <int M>
__device__ __forceinline__ void st_words(uint64_t* p, const uint64_t (&v)[M]) {
  if constexpr (M == 1) {
    p[0] = v[0];
  } else {
#pragma unroll
    for (int i = 0; i < M / 2; ++i)
      reinterpret_cast<ulonglong2*>(p)[i] = make_ulonglong2(v[2 * i], v[2 * i + 1]);
  }
}

// Faulty value of the injection element for word w of the tile.
__device__ __forceinline__ uint64_t inj_value(const SweepArgs& a, const InjRec& inj, uint32_t w) {
  const uint32_t x = inj.elem;
  if (inj.mode == 0) return ~a.good[(uint64_t)x * 32 + w];
  const uint64_t sv = inj.value ? ~0ull : 0ull;
  if (inj.pin == 0) return sv;
  const uint8_t t = a.type[x];
  const uint32_t f0 = a.fi_off[x];
  uint32_t nf = a.fi_off[x + 1] - f0;
  if (t == G_INV || t == G_CLKBUF || t == G_PO) nf = 1;
  uint64_t in[4] = {0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if ((uint32_t)k < nf) in[k] = a.good[(uint64_t)a.fi_idx[f0 + k] * 32 + w];
  const uint32_t pk = inj.pin - 1;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if ((uint32_t)k == pk) in[k] = sv;
  return eval_word(t, nf, in[0], in[1], in[2], in[3]);
}

template <int M>
__global__ void __launch_bounds__(512) k_sweep(SweepArgs a) {
  extern __shared__ __align__(16) uint64_t vals[];  // [max_live][M]
  __shared__ unsigned long long acc[M];
  __shared__ int s_item;
  const int tid = threadIdx.x, nth = blockDim.x;
  const uint32_t n_items = a.n_list * a.subtiles;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(a.queue, 1);
    if (tid < M) acc[tid] = 0ull;
    __syncthreads();
    const uint32_t item = (uint32_t)s_item;
    if (item >= n_items) return;
    const uint32_t li = item / a.subtiles;
    const uint32_t w0 = (item % a.subtiles) * M;
    const uint32_t si = a.list ? a.list[li] : li;
    const InjRec inj = a.inj[si];
    const uint32_t x = inj.elem;
    const uint32_t L0 = a.level[x] + 1;
    const uint32_t xmeta = a.meta[x];
    // Values live at the start level come from the good machine, except the
    // injection element itself.
    if (L0 <= a.max_gate_level) {
      const uint32_t i1 = a.li_off[L0 + 1];
      for (uint32_t i = a.li_off[L0] + tid; i < i1; i += nth) {
        const uint32_t e = a.li_elem[i];
        const uint32_t slot = a.meta[e] & kMetaSlotMask;
        uint64_t v[M];
        if (e == x) {
#pragma unroll
          for (int m = 0; m < M; ++m) v[m] = inj_value(a, inj, w0 + m);
        } else {
          ld_words<M>(a.good + (uint64_t)e * 32 + w0, v);
        }
        st_words<M>(vals + (size_t)slot * M, v);
      }
    }
    if (tid < M && ((xmeta & kMetaPo) || a.type[x] == G_PO)) {
      const uint32_t w = w0 + tid;
      acc[tid] = inj_value(a, inj, w) ^ a.good[(uint64_t)x * 32 + w];
    }
    __syncthreads();
    uint64_t pacc[M];
#pragma unroll
    for (int m = 0; m < M; ++m) pacc[m] = 0ull;
    for (uint32_t L = L0; L <= a.max_gate_level; ++L) {
      const uint32_t lo = a.level_off[L], hi = a.level_off[L + 1];
      for (uint32_t g = lo + tid; g < hi; g += nth) {
        const uint32_t mt = a.meta[g];
        const uint4 fs = a.fslot[g];
        const uint32_t t = (mt >> kMetaTypeShift) & 15u;
        const uint32_t nf = ((mt >> kMetaNfShift) & 3u) + 1u;
        uint64_t i0[M], i1[M], i2[M], i3[M];
        ld_words<M>(vals + (size_t)fs.x * M, i0);
        if (nf > 1) ld_words<M>(vals + (size_t)fs.y * M, i1);
        if (nf > 2) ld_words<M>(vals + (size_t)fs.z * M, i2);
        if (nf > 3) ld_words<M>(vals + (size_t)fs.w * M, i3);
        uint64_t r[M];
#pragma unroll
        for (int m = 0; m < M; ++m) r[m] = eval_word(t, nf, i0[m], i1[m], i2[m], i3[m]);
        if (mt & kMetaHasSlot) st_words<M>(vals + (size_t)(mt & kMetaSlotMask) * M, r);
        if (mt & kMetaPo) {
          uint64_t gv[M];
          ld_words<M>(a.good + (uint64_t)g * 32 + w0, gv);
#pragma unroll
          for (int m = 0; m < M; ++m) pacc[m] |= r[m] ^ gv[m];
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int m = 0; m < M; ++m)
      if (pacc[m]) atomicOr(&acc[m], (unsigned long long)pacc[m]);
    __syncthreads();
    if (tid < M) a.out[(uint64_t)si * 32 + w0 + tid] = acc[tid];
  }
}

// ---------------------------------------------------------------- FFR tracing
// Bits where flipping input `pin` of element p flips p's output, for bitwise
// gate types (MUX never reaches this path).
__device__ __forceinline__ uint64_t local_sens(const FfrArgs& a, uint32_t p, uint32_t pin,
                                               uint32_t lane) {
  const uint8_t t = a.type[p];
  if (t == G_XOR || t == G_XNOR) return ~0ull;
  if (t == G_INV || t == G_CLKBUF || t == G_PO) return pin == 0 ? ~0ull : 0ull;
  if (t == G_MUX || t == G_PI) return 0ull;
  const bool orf = (t == G_OR || t == G_NOR);
  const uint32_t f0 = a.fi_off[p], f1 = a.fi_off[p + 1];
  uint64_t s = ~0ull;
  for (uint32_t k = f0; k < f1; ++k) {
    if (k - f0 == pin) continue;
    const uint64_t g = a.good[(uint64_t)a.fi_idx[k] * 32 + lane];
    s &= orf ? ~g : g;
  }
  return s;
}

__device__ __forceinline__ void record(unsigned long long* count, unsigned long long* first,
                                       uint8_t* lastflag, uint32_t f, uint64_t D, uint32_t w,
                                       uint32_t bits, uint32_t W, uint32_t lane) {
  const unsigned ball = __ballot_sync(0xFFFFFFFFu, D != 0ull);
  const unsigned cnt = __reduce_add_sync(0xFFFFFFFFu, (unsigned)__popcll(D));
  if (ball) {
    const int fl = __ffs(ball) - 1;
    if ((int)lane == fl) {
      // lowest pattern index in the lowest detecting word: highest set bit
      const unsigned long long idx =
          (unsigned long long)w * 64ull + bits - 64ull + (unsigned long long)__clzll((long long)D);
      atomicMin(&first[f], idx);
      atomicAdd(&count[f], (unsigned long long)cnt);
    }
  }
  if (w == W - 1) lastflag[f] = D != 0ull;
}

__global__ void __launch_bounds__(256) k_ffr(FfrArgs a) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t n = a.n_list;
  if (warp >= n) return;
  const uint32_t ri = a.list ? a.list[warp] : warp;
  const RootRec rr = a.roots[ri];
  const uint32_t w = a.tile * 32 + lane;
  const uint32_t bits = round_bits(a.P, a.W, w);
  const uint64_t mask = bits_mask(bits);
  uint64_t obs;
  if (rr.obs == kObsOne)
    obs = ~0ull;
  else if (rr.obs == kObsZero)
    obs = 0ull;
  else
    obs = a.obs[(uint64_t)rr.obs * 32 + lane];
  obs &= mask;
  const uint64_t tile_first = (uint64_t)a.tile * 32 * 64;
  a.sens[(uint64_t)rr.root * 32 + lane] = ~0ull;
  for (uint32_t i = rr.mem_begin; i < rr.mem_end; ++i) {
    const MemberRec m = a.members[i];
    const uint64_t sp = a.sens[(uint64_t)m.p * 32 + lane];
    a.sens[(uint64_t)m.e * 32 + lane] = sp & local_sens(a, m.p, m.pin, lane);
  }
  for (uint32_t i = rr.flt_begin; i < rr.flt_end; ++i) {
    const TracedRec tr = a.traced[i];
    if (a.drop && a.first[tr.fault] < tile_first) continue;  // dropped earlier
    uint64_t s, gv;
    if (tr.pin == 0) {
      s = a.sens[(uint64_t)tr.elem * 32 + lane];
      gv = a.good[(uint64_t)tr.elem * 32 + lane];
    } else {
      s = a.sens[(uint64_t)tr.elem * 32 + lane] & local_sens(a, tr.elem, tr.pin - 1, lane);
      gv = a.good[(uint64_t)a.fi_idx[a.fi_off[tr.elem] + tr.pin - 1] * 32 + lane];
    }
    const uint64_t sv = tr.value ? ~0ull : 0ull;
    const uint64_t D = s & (gv ^ sv) & obs;
    record(a.count, a.first, a.lastflag, tr.fault, D, w, bits, a.W, lane);
  }
}

__global__ void __launch_bounds__(256) k_exact(ExactArgs a) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= a.n_exact) return;
  const uint32_t j = a.list ? a.list[warp] : warp;
  const uint32_t f = a.exact_fault[j];
  const uint64_t tile_first = (uint64_t)a.tile * 32 * 64;
  if (a.drop && a.first[f] < tile_first) return;
  const uint32_t w = a.tile * 32 + lane;
  const uint32_t bits = round_bits(a.P, a.W, w);
  const uint64_t mask = bits_mask(bits);
  const uint64_t D = a.out[(uint64_t)(a.first_sweep + j) * 32 + lane] & mask;
  record(a.count, a.first, a.lastflag, f, D, w, bits, a.W, lane);
}

__global__ void k_init_results(unsigned long long* count, unsigned long long* first,
                               uint8_t* lastflag, uint32_t F) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x) {
    count[i] = 0ull;
    first[i] = ~0ull;
    lastflag[i] = 0;
  }
}

// Keeps the roots that still carry an undetected traced fault and emits the
// sweep each of them needs; keeps undetected exact faults and their sweeps.
// Warp-aggregated appends: one atomic per warp and output list.
__global__ void k_drop(DropArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  const bool root_part = i < a.n_in_pad;  // uniform per warp (n_in_pad % 32 == 0)
  bool keep = false, sweep = false;
  uint32_t id = 0, sw = 0;
  if (root_part) {
    if (i < a.n_in) {
      id = a.in_list ? a.in_list[i] : i;
      const RootRec rr = a.roots[id];
      for (uint32_t k = rr.flt_begin; k < rr.flt_end && !keep; ++k)
        keep = a.count[a.traced[k].fault] == 0ull;
      sweep = keep && rr.obs != kObsOne && rr.obs != kObsZero;
      sw = rr.obs;
    }
  } else {
    const uint32_t j = i - a.n_in_pad;
    if (j < a.n_exact_in) {
      id = a.exact_in ? a.exact_in[j] : j;
      keep = a.count[a.exact_fault[id]] == 0ull;
      sweep = keep;
      sw = a.first_exact_sweep + id;
    }
  }
  const unsigned bk = __ballot_sync(0xFFFFFFFFu, keep);
  const unsigned bs = __ballot_sync(0xFFFFFFFFu, sweep);
  uint32_t base_k = 0, base_s = 0;
  if (lane == 0) {
    if (bk) base_k = atomicAdd(&a.n_out[root_part ? 0 : 2], (uint32_t)__popc(bk));
    if (bs) base_s = atomicAdd(&a.n_out[1], (uint32_t)__popc(bs));
  }
  base_k = __shfl_sync(0xFFFFFFFFu, base_k, 0);
  base_s = __shfl_sync(0xFFFFFFFFu, base_s, 0);
  if (keep) (root_part ? a.out_roots : a.out_exact)[base_k + __popc(bk & lt)] = id;
  if (sweep) a.out_sweeps[base_s + __popc(bs & lt)] = sw;
}

}  // namespace

void launch_good_level(const GoodArgs& a, cudaStream_t s) {
  const uint64_t n = (uint64_t)(a.hi - a.lo) * a.W_pad;
  if (n == 0) return;
  const int threads = 256;
  uint64_t blocks = (n + threads - 1) / threads;
  if (blocks > 148ull * 64) blocks = 148ull * 64;
  k_good_level<<<(unsigned)blocks, threads, 0, s>>>(a);
}

cudaError_t sweep_set_smem(int M, size_t smem) {
  switch (M) {
    case 1: return cudaFuncSetAttribute(k_sweep<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    case 2: return cudaFuncSetAttribute(k_sweep<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    case 4: return cudaFuncSetAttribute(k_sweep<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    case 8: return cudaFuncSetAttribute(k_sweep<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  return cudaErrorInvalidValue;
}

cudaError_t sweep_occupancy(int M, int threads, size_t smem, int* blocks_per_sm) {
  switch (M) {
    case 1: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_sweep<1>, threads, smem);
    case 2: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_sweep<2>, threads, smem);
    case 4: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_sweep<4>, threads, smem);
    case 8: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_sweep<8>, threads, smem);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_sweep(int M, int threads, int blocks, size_t smem, const SweepArgs& a,
                         cudaStream_t s) {
  switch (M) {
    case 1: k_sweep<1><<<blocks, threads, smem, s>>>(a); break;
    case 2: k_sweep<2><<<blocks, threads, smem, s>>>(a); break;
    case 4: k_sweep<4><<<blocks, threads, smem, s>>>(a); break;
    case 8: k_sweep<8><<<blocks, threads, smem, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

void launch_ffr(const FfrArgs& a, cudaStream_t s) {
  if (a.n_list == 0) return;
  const int threads = 256;
  const uint64_t blocks = ((uint64_t)a.n_list * 32 + threads - 1) / threads;
  k_ffr<<<(unsigned)blocks, threads, 0, s>>>(a);
}

void launch_exact(const ExactArgs& a, cudaStream_t s) {
  if (a.n_exact == 0) return;
  const int threads = 256;
  const uint64_t blocks = ((uint64_t)a.n_exact * 32 + threads - 1) / threads;
  k_exact<<<(unsigned)blocks, threads, 0, s>>>(a);
}

void launch_init_results(unsigned long long* count, unsigned long long* first, uint8_t* lastflag,
                         uint32_t F, cudaStream_t s) {
  if (F == 0) return;
  k_init_results<<<(F + 255) / 256 > 4096 ? 4096 : (F + 255) / 256, 256, 0, s>>>(count, first,
                                                                               lastflag, F);
}

void launch_drop(const DropArgs& a, cudaStream_t s) {
  const uint64_t n = (uint64_t)a.n_in_pad + a.n_exact_in;
  if (n == 0) return;
  k_drop<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
}

}  // namespace fsimb
