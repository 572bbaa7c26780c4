// B200 (sm_100a) kernels of the stuck-at fault simulator.
//
//   k_good_level   good machine, one launch per level, one thread per
//                  (element, word); warps cover the 32 words of a tile so every
//                  fanin read is one coalesced 256-byte segment.
//   k_sweep<M>     persistent: each CTA pulls (sweep, M-word subtile) items from
//                  a device work counter and re-simulates the levels above the
//                  injection point with all live values in shared memory
//                  (slots and a bank-conflict-free order chosen on the host;
//                  gate records staged per level by TMA bulk copies).  Writes
//                  the OR over POs of (faulty ^ good) per word.
//   k_sweep_wide<M> the same sweep for circuits whose live values do not
//                  fit in shared memory: values in a per-CTA region of global
//                  memory indexed by element.
//   k_ffr          one warp per FFR root, lanes = the 32 words of a tile:
//                  backward critical-path tracing inside the FFR and the
//                  per-fault detection word, count and first pattern.
//   k_exact        the same epilogue for faults simulated by an exact sweep.
//   k_drop         fault dropping: warp-aggregated stream compaction of the
//                  roots / sweeps that still carry faults below the N-detect
//                  limit.
//
// Word semantics follow fsim/simulation.cpp: gates act on whole 64-bit words
// (fsim/simulation.cpp:979-1124), the last round keeps its high bits until
// the PO comparison masks them (fsim/simulation.cpp:94-102, 174-178), and a
// detecting bit b of round rd with `bits` valid bits is pattern
// rd*64 + bits-1-b.
#include "fsimb_kernels.cuh"

#include <algorithm>

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

// ---------------------------------------------------------------- TMA bulk staging
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// One thread arms the barrier for `bytes` and starts a bulk copy (no
// multicast) of `bytes` from global to this CTA's shared memory.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  if (bytes == 0) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
    return;
  }
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the barrier's phase `parity` for at most limit_ns nanoseconds of
// the global timer (and at most 2^26 polls); false if it gave up, so the
// caller reports an error instead of hanging.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < (1u << 26); ++it) {
    if (mbar_try(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
  return false;
}

// Index of the last prefix entry <= x (prefix[0] = 0, n entries).
__device__ __forceinline__ uint32_t find_prefix(const unsigned long long* prefix, uint32_t n,
                                                unsigned long long x) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (prefix[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------- sweep
// Per-circuit pointers a sweep item reads (one circuit, one tile).
struct SweepView {
  const uint4* blob;       // level blocks of gate records (fsimb_plan.h)
  const uint4* lvl;        // LevelDesc per level
  const uint32_t* level;   // element -> level
  const uint32_t* li_off;
  const uint32_t* li;      // (element, slot) pairs
  const uint32_t* fi_off;
  const uint32_t* fi_idx;
  const uint8_t* type;
  const uint64_t* good;    // tile [N][32]
  uint32_t max_gate_level;
};

// Faulty value of the injection element for word w of the tile.
template <class V>
__device__ __forceinline__ uint64_t inj_value(const V& a, const InjRec& inj, uint32_t w) {
  const uint32_t x = inj.elem;
  if (!(inj.mode & kInjStuck)) return ~a.good[(uint64_t)x * 32 + w];
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
__device__ __forceinline__ void lds_chunk(const uint64_t* vals, uint32_t slot, int h, uint64_t (&v)[2]) {
  if constexpr (M == 1) {
    v[0] = vals[slot];
  } else {
    const ulonglong2 q = *reinterpret_cast<const ulonglong2*>(vals + (size_t)slot * M + 2 * h);
    v[0] = q.x;
    v[1] = q.y;
  }
}

template <int M>
__device__ __forceinline__ void sts_chunk(uint64_t* vals, uint32_t slot, int h, const uint64_t (&v)[2]) {
  if constexpr (M == 1)
    vals[slot] = v[0];
  else
    *reinterpret_cast<ulonglong2*>(vals + (size_t)slot * M + 2 * h) = make_ulonglong2(v[0], v[1]);
}

template <int M>
using PoAcc = uint64_t[(M >= 2) ? M / 2 : 1][(M >= 2) ? 2 : 1];

// ---- plain records: one body per family and fan-in (fsimb_plan.h plain_body)
// Slot chunk h of the value at byte offset `off` (slot * 8M).
template <int M>
__device__ __forceinline__ void ldo(const char* vb, uint32_t off, int h, uint64_t (&v)[2]) {
  if constexpr (M == 1) {
    v[0] = *reinterpret_cast<const uint64_t*>(vb + off);
  } else {
    const ulonglong2 q = *reinterpret_cast<const ulonglong2*>(vb + off + 16 * h);
    v[0] = q.x;
    v[1] = q.y;
  }
}
template <int M>
__device__ __forceinline__ void sto(char* vb, uint32_t off, int h, const uint64_t (&v)[2]) {
  if constexpr (M == 1)
    *reinterpret_cast<uint64_t*>(vb + off) = v[0];
  else
    *reinterpret_cast<ulonglong2*>(vb + off + 16 * h) = make_ulonglong2(v[0], v[1]);
}

// A plain record (fsimb_plan.h plain_rec) of body B on all M words.  B = 0:
// one input, io ^ a; 1 / 3: AND family with 2 / 3 inputs,
// io ^ AND(in ^ ii); 2 / 4: XOR family with 2 / 3 inputs, io ^ XOR(in).
// The inversions come from the class code: within the AND family the codes
// run AND, NAND, OR, NOR, so ii is bit 1 of the offset and io the XOR of
// its two bits; elsewhere io is bit 0 of the code.
template <int M, int B>
__device__ __forceinline__ void plain_body(char* vb, const uint2 r, int pl) {
  constexpr int C = (M >= 2) ? M / 2 : 1;
  constexpr int VC = (M >= 2) ? 2 : 1;
  constexpr int NF = B == 0 ? 1 : (B <= 2 ? 2 : 3);
  constexpr uint32_t SB = 8u * M;
  const uint32_t cls = r.y >> 28;
  uint32_t io_bit, ii_bit = 0;
  if constexpr (B == 1 || B == 3) {
    const uint32_t rel = cls - (B == 1 ? (uint32_t)kPAnd2 : (uint32_t)kPAnd3);
    ii_bit = (rel >> 1) & 1u;
    io_bit = (rel ^ (rel >> 1)) & 1u;
  } else {
    io_bit = cls & 1u;
  }
  const uint64_t ii = 0ull - (uint64_t)ii_bit, io = 0ull - (uint64_t)io_bit;
  const uint32_t o0 = (r.x & 0x7FFFu) * SB;
  const uint32_t o1 = ((r.x >> 15) & 0x7FFFu) * SB;
  const uint32_t o2 = (__funnelshift_r(r.x, r.y, 30) & 0x7FFFu) * SB;
  const uint32_t oo = ((r.y >> 13) & 0x7FFFu) * SB;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int h = (C == 1) ? 0 : (pl + c) % C;
    uint64_t a[2], b[2] = {0, 0}, d[2] = {0, 0}, o[2];
    ldo<M>(vb, o0, h, a);
    if constexpr (NF > 1) ldo<M>(vb, o1, h, b);
    if constexpr (NF > 2) ldo<M>(vb, o2, h, d);
#pragma unroll
    for (int v = 0; v < VC; ++v) {
      if constexpr (B == 0)
        o[v] = a[v] ^ io;
      else if constexpr (B == 1)
        o[v] = ((a[v] ^ ii) & (b[v] ^ ii)) ^ io;
      else if constexpr (B == 2)
        o[v] = a[v] ^ b[v] ^ io;
      else if constexpr (B == 3)
        o[v] = ((a[v] ^ ii) & (b[v] ^ ii) & (d[v] ^ ii)) ^ io;
      else
        o[v] = a[v] ^ b[v] ^ d[v] ^ io;
    }
    sto<M>(vb, oo, h, o);
  }
}

template <int M>
__device__ __forceinline__ void plain_dispatch(char* vb, const uint2 r, int pl) {
  // Records are grouped by body on the host, so a warp mostly takes one
  // path.  A chain of unsigned range tests on the class code, the
  // three-input AND family first, costs fewer instructions per record than
  // a switch over the classes.
  const uint32_t cls = r.y >> 28;
  if (cls - kPAnd3 < 4u)
    plain_body<M, 3>(vb, r, pl);
  else if (cls < kPAnd2)
    plain_body<M, 0>(vb, r, pl);
  else if (cls - kPAnd2 < 4u)
    plain_body<M, 1>(vb, r, pl);
  else if (cls - kPXor3 < 2u)
    plain_body<M, 4>(vb, r, pl);
  else if (cls - kPXor2 < 2u)
    plain_body<M, 2>(vb, r, pl);  // else kPNop
}

// ---- wide records (PO drivers, MUX, four inputs): runtime type and masks
// One gate of a known class (family F, fan-in NF) on all M words of the item:
// loads of the fanin chunks, the gate function, the store and the PO
// difference.  F = 0: io ^ AND(in ^ ii) covers AND, NAND, OR, NOR, INV and
// CLKBUF; F = 1: io ^ XOR(in) covers XOR and XNOR; F = 2: MUX.
template <int M, int F, int NF>
__device__ __forceinline__ void gate_body(uint64_t* vals, const uint4 q, uint32_t meta, int pl,
                                          const uint64_t* good_row, PoAcc<M>& pacc) {
  constexpr int C = (M >= 2) ? M / 2 : 1;
  constexpr int VC = (M >= 2) ? 2 : 1;
  const uint64_t ii = (meta & kRecIi) ? ~0ull : 0ull;
  const uint64_t io = (meta & kRecIo) ? ~0ull : 0ull;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int h = (pl + c) % C;
    uint64_t i0[2], i1[2] = {0, 0}, i2[2] = {0, 0}, i3[2] = {0, 0};
    lds_chunk<M>(vals, q.x & 0xFFFFu, h, i0);
    if constexpr (NF > 1) lds_chunk<M>(vals, q.x >> 16, h, i1);
    if constexpr (NF > 2) lds_chunk<M>(vals, q.y & 0xFFFFu, h, i2);
    if constexpr (NF > 3) lds_chunk<M>(vals, q.y >> 16, h, i3);
    uint64_t r[2];
#pragma unroll
    for (int v = 0; v < VC; ++v) {
      uint64_t x;
      if constexpr (F == 0) {
        x = i0[v] ^ ii;
        if constexpr (NF > 1) x &= i1[v] ^ ii;
        if constexpr (NF > 2) x &= i2[v] ^ ii;
        if constexpr (NF > 3) x &= i3[v] ^ ii;
        x ^= io;
      } else if constexpr (F == 1) {
        x = i0[v];
        if constexpr (NF > 1) x ^= i1[v];
        if constexpr (NF > 2) x ^= i2[v];
        if constexpr (NF > 3) x ^= i3[v];
        x ^= io;
      } else {
        // (s & b) | (a & !s) with a logical not (fsim/simulation.cpp:1056)
        x = (i2[v] & i1[v]) | (i0[v] & (uint64_t)(i2[v] == 0));
      }
      r[v] = x;
    }
    if (meta & kRecHasSlot) sts_chunk<M>(vals, q.z & 0xFFFFu, h, r);
    if (meta & kRecPo) {
#pragma unroll
      for (int v = 0; v < VC; ++v) pacc[c][v] |= r[v] ^ good_row[VC * h + v];
    }
  }
}

// Any other class (rare combinations): word-by-word generic evaluation.
template <int M>
__device__ __forceinline__ void gate_generic(uint64_t* vals, const uint4 q, uint32_t meta, int pl,
                                             const uint64_t* good_row, PoAcc<M>& pacc) {
  constexpr int C = (M >= 2) ? M / 2 : 1;
  constexpr int VC = (M >= 2) ? 2 : 1;
  const uint32_t t = meta & kRecTypeMask;
  const uint32_t nf = ((meta >> kRecNfShift) & 3u) + 1u;
  for (int c = 0; c < C; ++c) {
    const int h = (pl + c) % C;
    uint64_t i0[2], i1[2] = {0, 0}, i2[2] = {0, 0}, i3[2] = {0, 0};
    lds_chunk<M>(vals, q.x & 0xFFFFu, h, i0);
    if (nf > 1) lds_chunk<M>(vals, q.x >> 16, h, i1);
    if (nf > 2) lds_chunk<M>(vals, q.y & 0xFFFFu, h, i2);
    if (nf > 3) lds_chunk<M>(vals, q.y >> 16, h, i3);
    uint64_t r[2];
    for (int v = 0; v < VC; ++v) r[v] = eval_word(t, nf, i0[v], i1[v], i2[v], i3[v]);
    if (meta & kRecHasSlot) sts_chunk<M>(vals, q.z & 0xFFFFu, h, r);
    if (meta & kRecPo)
      for (int v = 0; v < VC; ++v) pacc[c][v] |= r[v] ^ good_row[VC * h + v];
  }
}

template <int M>
__device__ __forceinline__ void gate_dispatch(uint64_t* vals, const uint4 q, int pl,
                                              const uint64_t* good_row, PoAcc<M>& pacc) {
  const uint32_t meta = q.z >> 16;
  switch ((meta >> kRecClassShift) & 15u) {  // dense class index from the host (gate_class)
    case 0: gate_body<M, 0, 1>(vals, q, meta, pl, good_row, pacc); break;
    case 1: gate_body<M, 0, 2>(vals, q, meta, pl, good_row, pacc); break;
    case 2: gate_body<M, 0, 3>(vals, q, meta, pl, good_row, pacc); break;
    case 3: gate_body<M, 0, 4>(vals, q, meta, pl, good_row, pacc); break;
    case 4: gate_body<M, 1, 2>(vals, q, meta, pl, good_row, pacc); break;
    case 5: gate_body<M, 1, 3>(vals, q, meta, pl, good_row, pacc); break;
    case 6: gate_body<M, 1, 4>(vals, q, meta, pl, good_row, pacc); break;
    case 7: gate_body<M, 2, 3>(vals, q, meta, pl, good_row, pacc); break;
    default: gate_generic<M>(vals, q, meta, pl, good_row, pacc); break;
  }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// M words per item, one thread per gate holding all M words.  Slots are
// M*8 bytes; a thread reads a slot as C = M/2 16-byte chunks (one 8-byte word
// for M = 1).  The host orders each level in groups of G = 16/M consecutive
// positions whose slots have distinct residues mod G (for every fanin and the
// output).  Within a phase of 8 lanes (16 for M = 1), lane l takes position
// (l % C) * G + l / C and reads chunk (l + i) % C at step i, so the 8 chunks a
// phase touches lie in 8 different bank quads: the loads and stores of a
// sweep are free of bank conflicts wherever the host found such groups.
//
// Each level's block of gate records is staged into one of two shared-memory
// buffers by a TMA bulk copy issued two levels ahead (one elected thread,
// mbarrier completion, waits bounded in time); a block larger than a buffer
// reads the rest from global memory.
struct SweepCta {
  uint64_t* vals;     // [max_live][M]
  uint4* recbuf;      // [2][rec_buf]
  uint64_t* bars;     // [3] mbarriers: two staging buffers, one for the wait test
  unsigned long long* acc;
  uint32_t rec_buf;   // 16-byte units per staging buffer
  uint32_t uses;      // levels staged and consumed so far: use u goes through
                      // buffer u & 1 and completes that barrier's phase u >> 1
  uint64_t wait_ns;   // limit of one wait
  uint32_t test_stall;
};

template <int M>
__device__ __forceinline__ void sweep_cta_init(SweepCta& k, uint64_t* vals, uint32_t vals_bytes,
                                               uint32_t rec_buf, uint64_t* bars, unsigned long long* acc,
                                               uint64_t wait_ns, uint32_t test_stall) {
  k.vals = vals;
  k.recbuf = reinterpret_cast<uint4*>(reinterpret_cast<char*>(vals) + vals_bytes);
  k.bars = bars;
  k.acc = acc;
  k.rec_buf = rec_buf;
  k.uses = 0;
  k.wait_ns = wait_ns;
  k.test_stall = test_stall;
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init(&bars[2], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

// Thread 0 only: the block of level L into buffer b.
__device__ __forceinline__ void sweep_stage(SweepCta& k, const SweepView& v, uint32_t L, int b) {
  const uint4 d = v.lvl[L];
  const uint32_t n = min(d.w, k.rec_buf);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  bulk_load(k.recbuf + (size_t)b * k.rec_buf, v.blob + d.x, n * 16u, &k.bars[b]);
}

// Error path: thread 0 waits (bounded) for the n copies still in flight
// into this CTA's shared memory (uses u, u + 1, ...), so none lands after
// the CTA has exited.  A copy already waited for passes at once.
__device__ __forceinline__ void sweep_drain(SweepCta& k, uint32_t u, uint32_t n) {
  if (threadIdx.x == 0)
    for (uint32_t i = 0; i < n; ++i) mbar_wait(&k.bars[(u + i) & 1u], ((u + i) >> 1) & 1u, k.wait_ns);
  __syncthreads();
}

// One item: the levels above the injection element for M words starting at
// word w0 of the tile; writes the OR of PO differences to out_row[w0..w0+M).
// Returns false (on every thread) if a bounded wait gave up.
template <int M>
__device__ __forceinline__ bool sweep_item(SweepCta& k, const SweepView& v, const InjRec inj, uint32_t w0,
                                           uint64_t* out_row) {
  constexpr int C = (M >= 2) ? M / 2 : 1;   // chunks per slot
  constexpr int VC = (M >= 2) ? 2 : 1;      // words per chunk
  constexpr int G = 16 / M;                 // residue group size
  constexpr int PH = (M == 1) ? 16 : 8;     // lanes per shared-memory phase
  const int tid = threadIdx.x, nth = blockDim.x;
  const int pl = tid & (PH - 1);
  const uint32_t my_off = (uint32_t)((tid & ~(PH - 1)) + ((M >= 2) ? (pl % C) * G + pl / C : pl));
  const uint32_t Lmax = v.max_gate_level;
  uint64_t* vals = k.vals;
  char* vb = reinterpret_cast<char*>(vals);
  const uint32_t x = inj.elem;
  const uint32_t L0 = v.level[x] + 1;
  if (tid < M) k.acc[tid] = 0ull;
  const uint32_t n_out = L0 > Lmax ? 0u : (L0 + 1 <= Lmax ? 2u : 1u);  // copies issued ahead
  if (tid == 0) {
    if (n_out > 0) sweep_stage(k, v, L0, (int)(k.uses & 1u));
    if (n_out > 1) sweep_stage(k, v, L0 + 1, (int)((k.uses + 1) & 1u));
  }
  bool ok = true;
  if (k.test_stall) {
    // test hook: wait on a barrier that no copy completes, so the wait runs
    // out and the item takes the error path
    k.test_stall = 0;
    if (tid == 0) ok = mbar_wait(&k.bars[2], 0, k.wait_ns);
  }
  if (L0 <= Lmax) {
    // Values live at the start level come from the good machine (copied
    // asynchronously, four list entries in flight per thread), except the
    // injection element itself.
    const uint32_t i1 = v.li_off[L0 + 1];
    const uint2* li = reinterpret_cast<const uint2*>(v.li);
    for (uint32_t i = v.li_off[L0] + tid; i < i1; i += 4 * nth) {
      uint2 es[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) es[j] = (i + j * nth < i1) ? li[i + j * nth] : make_uint2(0xFFFFFFFFu, 0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (es[j].x == 0xFFFFFFFFu) continue;
        uint64_t* dst = vals + (size_t)es[j].y * M;
        if (es[j].x == x) {
#pragma unroll
          for (int m = 0; m < M; ++m) dst[m] = inj_value(v, inj, w0 + m);
        } else {
          const uint64_t* src = v.good + (uint64_t)es[j].x * 32 + w0;
          if constexpr (M == 1) {
            cp_async8(dst, src);
          } else {
#pragma unroll
            for (int q = 0; q < M / 2; ++q) cp_async16(dst + 2 * q, src + 2 * q);
          }
        }
      }
    }
    cp_async_wait_all();
  }
  if (tid < M && (inj.mode & kInjReachesPo))
    k.acc[tid] = inj_value(v, inj, w0 + tid) ^ v.good[(uint64_t)x * 32 + w0 + tid];
  if (__syncthreads_or(!ok)) {
    sweep_drain(k, k.uses, n_out);
    return false;
  }
  PoAcc<M> pacc;
#pragma unroll
  for (int c = 0; c < C; ++c)
#pragma unroll
    for (int q = 0; q < VC; ++q) pacc[c][q] = 0ull;
  for (uint32_t L = L0; L <= Lmax; ++L) {
    const uint32_t u = k.uses;
    const int b = (int)(u & 1u);
    const uint4 desc = v.lvl[L];  // issued before the wait, used after it
    ok = mbar_wait(&k.bars[b], (u >> 1) & 1u, k.wait_ns);
    if (ok) {
      const char* sb = reinterpret_cast<const char*>(k.recbuf + (size_t)b * k.rec_buf);
      const char* gb = reinterpret_cast<const char*>(v.blob + desc.x);
      const uint32_t staged = min(desc.w, k.rec_buf) * 16u;
      const uint32_t np = desc.y, n = desc.y + desc.z;
      const uint32_t wide0 = (np + 1) / 2 * 16;
      // Plain records from the staging buffer, then the rest of the plain
      // part from global memory, then the wide records: three loops
      // without a per-record choice of source cost fewer instructions than
      // one loop that picks the source and the record kind per position.
      const uint32_t ns = min(np, staged / 8u);
      uint32_t p = my_off;
      for (; p < ns; p += nth) plain_dispatch<M>(vb, *reinterpret_cast<const uint2*>(sb + (size_t)p * 8), pl);
      for (; p < np; p += nth) plain_dispatch<M>(vb, *reinterpret_cast<const uint2*>(gb + (size_t)p * 8), pl);
      for (; p < n; p += nth) {
        const uint32_t byte = wide0 + (p - np) * 16;
        uint4 q;
        if (byte < staged)
          q = *reinterpret_cast<const uint4*>(sb + byte);
        else
          q = *reinterpret_cast<const uint4*>(gb + byte);
        gate_dispatch<M>(vals, q, pl, v.good + (uint64_t)q.w * 32 + w0, pacc);
      }
    }
    if (__syncthreads_or(!ok)) {
      sweep_drain(k, u, L + 1 <= Lmax ? 2u : 1u);
      return false;
    }
    k.uses = u + 1;
    if (L + 2 <= Lmax && tid == 0) sweep_stage(k, v, L + 2, b);
  }
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int h = (pl + c) % C;
#pragma unroll
    for (int q = 0; q < VC; ++q)
      if (pacc[c][q]) atomicOr(&k.acc[VC * h + q], (unsigned long long)pacc[c][q]);
  }
  __syncthreads();
  if (tid < M) out_row[w0 + tid] = k.acc[tid];
  return true;
}

// Register caps: the CTA sizes up to sweep_max_threads(M) fit the register
// file, and 56 at M = 2 lets three 384-thread CTAs share an SM.
template <int M>
__global__ void __maxnreg__(M >= 8 ? 120 : (M >= 4 ? 72 : (M >= 2 ? 56 : 64))) k_sweep(SweepArgs a) {
  extern __shared__ __align__(16) uint64_t vals[];  // [max_live][M] | recbuf[2][rec_buf]
  __shared__ unsigned long long acc[M];
  __shared__ __align__(8) uint64_t bars[3];
  __shared__ int s_item;
  SweepCta k;
  sweep_cta_init<M>(k, vals, a.vals_bytes, a.rec_buf, bars, acc, a.wait_ns,
                    (a.wait_test && blockIdx.x == 0) ? 1u : 0u);
  const SweepView v{a.blob, a.lvl, a.level, a.li_off, a.li, a.fi_off, a.fi_idx, a.type, a.good,
                    a.max_gate_level};
  constexpr uint32_t subtiles = kTileWords / M;
  const uint32_t n_items = a.n_list * subtiles;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(a.queue, 1);
    __syncthreads();
    const uint32_t item = (uint32_t)s_item;
    __syncthreads();  // s_item is rewritten for the next item only after all have read it
    if (item >= n_items) return;
    const uint32_t li = item / subtiles;
    const uint32_t w0 = (item % subtiles) * M;
    const uint32_t si = a.list ? a.list[li] : li;
    if (!sweep_item<M>(k, v, a.inj[si], w0, a.out + (uint64_t)si * 32)) {
      if (threadIdx.x == 0) atomicExch(a.err, 1);
      return;
    }
  }
}

// Batch form: the circuits of one launch, each with its own work counter.
// Every CTA walks the circuits in order and takes (tile, sweep, subtile)
// items of each until its counter runs out, so items are consumed in
// circuit order as from one queue.  The loop index is uniform and the
// circuit fields come from the kernel parameters: the compiler keeps the
// pointers in uniform registers, as for k_sweep.
template <int M>
__global__ void __maxnreg__(M >= 8 ? 96 : (M >= 4 ? 72 : (M >= 2 ? 56 : 64)))
    k_sweep_batch(const __grid_constant__ BatchSweepParams p) {
  extern __shared__ __align__(16) uint64_t vals[];
  __shared__ unsigned long long acc[M];
  __shared__ __align__(8) uint64_t bars[3];
  __shared__ uint32_t s_item;
  SweepCta k;
  sweep_cta_init<M>(k, vals, p.vals_bytes, p.rec_buf, bars, acc, p.wait_ns, 0u);
  constexpr uint32_t subtiles = kTileWords / M;
  for (uint32_t ci = 0; ci < p.n_circ; ++ci) {
    const SweepCirc& c = p.c[ci];
    const uint32_t per_tile = c.n_sweeps * subtiles;
    for (;;) {
      if (threadIdx.x == 0) {
        const unsigned long long it = atomicAdd(p.queue + ci, 1ull);
        s_item = it < c.n_items ? (uint32_t)it : 0xFFFFFFFFu;
      }
      __syncthreads();
      const uint32_t item = s_item;
      __syncthreads();  // s_item is rewritten only after every thread read it
      if (item == 0xFFFFFFFFu) break;
      const uint32_t tile = item / per_tile;
      const uint32_t rem = item - tile * per_tile;
      const uint32_t si = rem / subtiles;
      const uint32_t w0 = (rem % subtiles) * M;
      const SweepView v{c.blob, c.lvl, c.level, c.li_off, c.li, c.fi_off, c.fi_idx, c.type,
                        c.good + (uint64_t)tile * c.N * 32, c.max_gate_level};
      if (!sweep_item<M>(k, v, c.inj[si], w0, c.out + ((uint64_t)tile * c.n_sweeps + si) * 32)) {
        if (threadIdx.x == 0) atomicExch(p.err, 1);
        return;
      }
    }
  }
}

// ---------------------------------------------------------------- wide circuits
// Sweep for circuits whose live values do not fit in shared memory: every
// CTA keeps the values of its item in its own region of global memory,
// indexed by element (gvals + block * N * M), which L2 mostly holds.  A
// fanin below the start level other than the injection element reads the
// good machine directly, so an item starts without copying live values.
// Threads take (element, word) pairs of a level; one barrier per level.
template <int M>
__global__ void __launch_bounds__(256) k_sweep_wide(SweepWideArgs a) {
  __shared__ unsigned long long acc[M];
  __shared__ uint32_t s_item;
  uint64_t* gv = a.gvals + (size_t)blockIdx.x * a.N * M;
  const uint32_t tid = threadIdx.x, nth = blockDim.x;
  const uint32_t m = tid % M, step = nth / M;
  constexpr uint32_t subtiles = kTileWords / M;
  const uint32_t n_items = a.n_list * subtiles;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(a.queue, 1);
    __syncthreads();
    const uint32_t item = s_item;
    __syncthreads();
    if (item >= n_items) return;
    const uint32_t li = item / subtiles;
    const uint32_t w0 = (item % subtiles) * M;
    const uint32_t si = a.list ? a.list[li] : li;
    const InjRec inj = a.inj[si];
    const uint32_t x = inj.elem;
    const uint32_t L0 = a.level[x] + 1;
    const uint32_t lo0 = L0 <= a.max_gate_level ? a.level_off[L0] : 0;
    if (tid < M) {
      const uint64_t fv = inj_value(a, inj, w0 + tid);
      gv[(size_t)x * M + tid] = fv;
      acc[tid] = (inj.mode & kInjReachesPo) ? fv ^ a.good[(uint64_t)x * 32 + w0 + tid] : 0ull;
    }
    __syncthreads();
    uint64_t pacc = 0;
    const uint32_t w = w0 + m;
    for (uint32_t L = L0; L <= a.max_gate_level; ++L) {
      const uint32_t lo = a.level_off[L], hi = a.level_off[L + 1];
      for (uint32_t e = lo + tid / M; e < hi; e += step) {
        const uint8_t fl = a.eflag[e];
        if (!(fl & 1u)) continue;
        const uint8_t t = a.type[e];
        const uint32_t f0 = a.fi_off[e];
        uint32_t nf = a.fi_off[e + 1] - f0;
        if (t == G_INV || t == G_CLKBUF || t == G_PO) nf = 1;
        uint64_t in[4] = {0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if ((uint32_t)q < nf) {
            const uint32_t f = a.fi_idx[f0 + q];
            in[q] = (f < lo0 && f != x) ? a.good[(uint64_t)f * 32 + w] : gv[(size_t)f * M + m];
          }
        }
        const uint64_t r = eval_word(t, nf, in[0], in[1], in[2], in[3]);
        gv[(size_t)e * M + m] = r;
        if (fl & 2u) pacc |= r ^ a.good[(uint64_t)e * 32 + w];
      }
      __syncthreads();
    }
    if (pacc) atomicOr(&acc[m], (unsigned long long)pacc);
    __syncthreads();
    if (tid < M) a.out[(uint64_t)si * 32 + w0 + tid] = acc[tid];
  }
}

// ---------------------------------------------------------------- FFR tracing
// Bits where flipping input `pin` of element p flips p's output, for bitwise
// gate types (MUX never reaches this path).
template <class V>
__device__ __forceinline__ uint64_t local_sens(const V& a, uint32_t p, uint32_t pin, uint32_t lane) {
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
  a.sens[(uint64_t)rr.root * 32 + lane] = ~0ull;
  for (uint32_t i = rr.mem_begin; i < rr.mem_end; ++i) {
    const MemberRec m = a.members[i];
    const uint64_t sp = a.sens[(uint64_t)m.p * 32 + lane];
    a.sens[(uint64_t)m.e * 32 + lane] = sp & local_sens(a, m.p, m.pin, lane);
  }
  for (uint32_t i = rr.flt_begin; i < rr.flt_end; ++i) {
    const TracedRec tr = a.traced[i];
    if (a.drop && a.count[tr.fault] >= a.n_detect) continue;  // dropped after an earlier tile
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
  if (a.drop && a.count[f] >= a.n_detect) return;  // dropped after an earlier tile
  const uint32_t w = a.tile * 32 + lane;
  const uint32_t bits = round_bits(a.P, a.W, w);
  const uint64_t mask = bits_mask(bits);
  const uint64_t D = a.out[(uint64_t)(a.first_sweep + j) * 32 + lane] & mask;
  record(a.count, a.first, a.lastflag, f, D, w, bits, a.W, lane);
}

// ---------------------------------------------------------------- batches
// The good-machine words and scratch of one circuit's tile, for the batched
// tracing kernels.
struct TileView {
  const uint8_t* type;
  const uint32_t* fi_off;
  const uint32_t* fi_idx;
  const uint64_t* good;
};

// One warp per (element, tile) of a level, over the circuits of the batch.
__global__ void __launch_bounds__(256) k_good_batch(const BatchCirc* circs, const BatchGoodSeg* segs,
                                                    uint32_t n_segs, unsigned long long n_units) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long unit = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (unit >= n_units) return;
  uint32_t lo = 0, hi = n_segs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (segs[mid].unit0 <= unit) lo = mid; else hi = mid;
  }
  const BatchGoodSeg sg = segs[lo];
  const BatchCirc& c = circs[sg.circ];
  const unsigned long long local = unit - sg.unit0;
  const uint32_t e = sg.lo + (uint32_t)(local / c.tiles);
  const uint32_t tile = (uint32_t)(local % c.tiles);
  const uint32_t w = tile * 32 + lane;
  const uint64_t base = (uint64_t)tile * c.N;
  const uint8_t t = c.type[e];
  uint64_t v;
  if (t == G_PI) {
    v = (w < c.W) ? c.pwords[(uint64_t)w * c.n_pi + e] : 0ull;
  } else {
    const uint32_t f0 = c.fi_off[e];
    uint32_t nf = c.fi_off[e + 1] - f0;
    if (t == G_INV || t == G_CLKBUF || t == G_PO) nf = 1;
    uint64_t in[4] = {0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if ((uint32_t)k < nf) in[k] = c.good[(base + c.fi_idx[f0 + k]) * 32 + lane];
    v = eval_word(t, nf, in[0], in[1], in[2], in[3]);
  }
  c.good[(base + e) * 32 + lane] = v;
}

// One warp per (circuit, tile, root): the k_ffr body on that circuit's tile.
__global__ void __launch_bounds__(256) k_ffr_batch(BatchUnits u, unsigned long long n_units) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long unit = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (unit >= n_units) return;
  const uint32_t ci = find_prefix(u.unit_prefix, u.n_circ, unit);
  const BatchCirc& c = u.circs[ci];
  const unsigned long long local = unit - u.unit_prefix[ci];
  const uint32_t tile = (uint32_t)(local / c.n_roots);
  const uint32_t ri = (uint32_t)(local % c.n_roots);
  const TileView tv{c.type, c.fi_off, c.fi_idx, c.good + (uint64_t)tile * c.N * 32};
  // compact sensitivities: slot i = members[i], slot n_members + r = root r
  uint64_t* sens = c.sens + (uint64_t)tile * c.n_slots * 32;
  const uint64_t* obsv = c.out + (uint64_t)tile * c.n_sweeps * 32;
  const RootRec rr = c.roots[ri];
  const uint32_t w = tile * 32 + lane;
  const uint32_t bits = round_bits(c.P, c.W, w);
  uint64_t obs = rr.obs == kObsOne ? ~0ull : rr.obs == kObsZero ? 0ull : obsv[(uint64_t)rr.obs * 32 + lane];
  obs &= bits_mask(bits);
  sens[(uint64_t)rr.slot * 32 + lane] = ~0ull;
  for (uint32_t i = rr.mem_begin; i < rr.mem_end; ++i) {
    const MemberRec m = c.members[i];
    sens[(uint64_t)i * 32 + lane] = sens[(uint64_t)m.p_slot * 32 + lane] & local_sens(tv, m.p, m.pin, lane);
  }
  for (uint32_t i = rr.flt_begin; i < rr.flt_end; ++i) {
    const TracedRec tr = c.traced[i];
    const uint64_t st = sens[(uint64_t)c.traced_slot[i] * 32 + lane];
    uint64_t sv, gv;
    if (tr.pin == 0) {
      sv = st;
      gv = tv.good[(uint64_t)tr.elem * 32 + lane];
    } else {
      sv = st & local_sens(tv, tr.elem, tr.pin - 1, lane);
      gv = tv.good[(uint64_t)c.fi_idx[c.fi_off[tr.elem] + tr.pin - 1] * 32 + lane];
    }
    const uint64_t D = sv & (gv ^ (tr.value ? ~0ull : 0ull)) & obs;
    record(c.count, c.first, c.lastflag, tr.fault, D, w, bits, c.W, lane);
  }
}

// One warp per (circuit, tile, exact fault).
__global__ void __launch_bounds__(256) k_exact_batch(BatchUnits u, unsigned long long n_units) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long unit = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (unit >= n_units) return;
  const uint32_t ci = find_prefix(u.unit_prefix, u.n_circ, unit);
  const BatchCirc& c = u.circs[ci];
  const unsigned long long local = unit - u.unit_prefix[ci];
  const uint32_t tile = (uint32_t)(local / c.n_exact);
  const uint32_t j = (uint32_t)(local % c.n_exact);
  const uint32_t w = tile * 32 + lane;
  const uint32_t bits = round_bits(c.P, c.W, w);
  const uint64_t D = c.out[((uint64_t)tile * c.n_sweeps + c.n_stem_sweeps + j) * 32 + lane] & bits_mask(bits);
  record(c.count, c.first, c.lastflag, c.exact_fault[j], D, w, bits, c.W, lane);
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
        keep = a.count[a.traced[k].fault] < a.n_detect;
      sweep = keep && rr.obs != kObsOne && rr.obs != kObsZero;
      sw = rr.obs;
    }
  } else {
    const uint32_t j = i - a.n_in_pad;
    if (j < a.n_exact_in) {
      id = a.exact_in ? a.exact_in[j] : j;
      keep = a.count[a.exact_fault[id]] < a.n_detect;
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

void launch_good_batch(const BatchCirc* circs, const BatchGoodSeg* segs, uint32_t n_segs,
                       unsigned long long n_units, cudaStream_t s) {
  if (!n_units) return;
  k_good_batch<<<(unsigned)((n_units * 32 + 255) / 256), 256, 0, s>>>(circs, segs, n_segs, n_units);
}

void launch_ffr_batch(const BatchUnits& u, unsigned long long n_units, cudaStream_t s) {
  if (!n_units) return;
  k_ffr_batch<<<(unsigned)((n_units * 32 + 255) / 256), 256, 0, s>>>(u, n_units);
}

void launch_exact_batch(const BatchUnits& u, unsigned long long n_units, cudaStream_t s) {
  if (!n_units) return;
  k_exact_batch<<<(unsigned)((n_units * 32 + 255) / 256), 256, 0, s>>>(u, n_units);
}

void launch_init_results_batch(unsigned long long* count, unsigned long long* first, uint8_t* lastflag,
                               uint64_t F, cudaStream_t s) {
  if (!F) return;
  const uint64_t blocks = std::min<uint64_t>((F + 255) / 256, 4096);
  k_init_results<<<(unsigned)blocks, 256, 0, s>>>(count, first, lastflag, (uint32_t)std::min<uint64_t>(F, 0xFFFFFFFFull));
}

#define FSIMB_SWEEP_BATCH_CASES(X) X(1) X(2) X(4) X(8)
cudaError_t sweep_batch_set_smem(int M, size_t smem) {
  switch (M) {
#define X(m) case m: return cudaFuncSetAttribute(k_sweep_batch<m>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    FSIMB_SWEEP_BATCH_CASES(X)
#undef X
  }
  return cudaErrorInvalidValue;
}

cudaError_t sweep_batch_occupancy(int M, int threads, size_t smem, int* blocks_per_sm) {
  switch (M) {
#define X(m) case m: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_sweep_batch<m>, threads, smem);
    FSIMB_SWEEP_BATCH_CASES(X)
#undef X
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_sweep_batch(int M, int threads, int blocks, size_t smem, const BatchSweepParams& p,
                               cudaStream_t s) {
  switch (M) {
#define X(m) case m: k_sweep_batch<m><<<blocks, threads, smem, s>>>(p); break;
    FSIMB_SWEEP_BATCH_CASES(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

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

cudaError_t launch_sweep_wide(int M, int blocks, const SweepWideArgs& a, cudaStream_t s) {
  switch (M) {
    case 1: k_sweep_wide<1><<<blocks, 256, 0, s>>>(a); break;
    case 2: k_sweep_wide<2><<<blocks, 256, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t sweep_wide_occupancy(int M, int* blocks_per_sm) {
  switch (M) {
    case 1: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_sweep_wide<1>, 256, 0);
    case 2: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_sweep_wide<2>, 256, 0);
  }
  return cudaErrorInvalidValue;
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
