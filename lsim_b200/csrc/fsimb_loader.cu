// Fast .ckt loader: host threads tokenize the text, the device builds the
// pin-slot table, the element order, the levels and both CSRs.  The result
// is the Netlist the host reader (fsimb_netlist.cpp) builds, field for
// field; any input that reader would reject, or whose levels are not sorted
// in element order, is handed back to it (parse_ckt_device returns false).
//
// Element order (fsim/simulation.cpp:718-751): the Kahn FIFO seeded with the
// PIs in id order, each element's successors appended in adjacency
// (insertion) order once their last in-edge is taken.  The FIFO is built
// here in waves: wave 0 holds the PIs; an element joins wave w+1 when its
// last predecessor is in wave w, and the FIFO lists the waves in turn.
// Within a wave the FIFO order is the order of (position of the last
// predecessor, index of its last edge to the element in that predecessor's
// adjacency list) -- the moment the FIFO appends the element.  One 64-bit
// atomicMax per edge gives that key; a per-wave count, scan and ordered
// emit place the wave.  POs take no part in the waves: they never trigger
// an element, and the reference moves them to the end in id order.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <memory>
#include <thread>

#include "fsimb_internal.h"
#include "fsimb_loader.h"

namespace fsimb {

namespace {

constexpr int kBlock = 256;

inline bool ws(char c) {
  return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\f' || c == '\v';
}

inline double ms_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

inline unsigned grid_for(uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + kBlock - 1) / kBlock, 148 * 64)); }

// Error bits a kernel sets when the input needs the host reader.
enum : uint32_t { kBadSink = 1, kTooManyInputs = 2, kMuxInputs = 4, kNoInput = 8 };

struct LoaderDev {
  DevBuf a, line_src, line_k, line_off, line_eoff, types;
  DevBuf indeg, wait, slot, esrc, outdeg, adj_off, line_key, line_key2, line_id, line_id2, line_ksorted,
      line_rsorted, line_rank, adj, key, pos, lev, front[2], cnt, offs, ctl;
  DevBuf tpg, order, type_t, level_t, fcount, fi_off, fi_idx, cons, fpin, fo_cnt, fo_off, fo_key,
      fo_key2, fo_val, fo_val2, fo_idx, fo_pin, temp;
  ~LoaderDev() {
    for (DevBuf* b : {&a, &line_src, &line_k, &line_off, &line_eoff, &types, &indeg, &wait, &slot, &esrc,
                      &outdeg, &adj_off, &line_key, &line_key2, &line_id, &line_id2, &line_ksorted,
                      &line_rsorted, &line_rank, &adj, &key, &pos, &lev, &front[0], &front[1], &cnt,
                      &offs, &ctl, &tpg, &order, &type_t, &level_t, &fcount, &fi_off, &fi_idx, &cons,
                      &fpin, &fo_cnt, &fo_off, &fo_key, &fo_key2, &fo_val, &fo_val2, &fo_idx, &fo_pin, &temp})
      b->release();
  }
};

// ctl words: [0] error bits, [1] POs reached, [2] max gate level, [3] next
// wave size, [4] levels not sorted.
struct Ctl {
  uint32_t err, po_reached, max_level, next_n, unsorted;
};

struct Dims {
  uint32_t N, nPI, nPO, nG;
};

__device__ __forceinline__ bool is_po(const Dims& d, uint32_t f) { return f >= d.nPI && f < d.nPI + d.nPO; }

// One thread per wire line: edges, in-degrees, last writer of each pin slot
// (fsim/simulation.cpp:684-711: a later write to a slot replaces an earlier
// one, every write counts an input).
__global__ void k_edges(Dims d, uint32_t W, const uint32_t* __restrict__ a, const uint32_t* __restrict__ line_src,
                        const uint32_t* __restrict__ line_k, const uint32_t* __restrict__ line_off,
                        const uint32_t* __restrict__ line_eoff, uint32_t* indeg, uint32_t* slot,
                        uint32_t* __restrict__ esrc, uint32_t* outdeg, Ctl* ctl) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
    const uint32_t src = line_src[w], k = line_k[w], off = line_off[w], e0 = line_eoff[w];
    if (k) atomicAdd(outdeg + src, k);
    for (uint32_t j = 0; j < k; ++j) {
      const uint32_t dst = a[off + 2 * j];
      uint32_t pin = a[off + 2 * j + 1];
      const uint32_t e = e0 + j;
      esrc[e] = src;
      if (dst >= d.N || dst < d.nPI || pin < 1 || pin > 5) {
        atomicOr(&ctl->err, kBadSink);
        continue;
      }
      if (pin == 5) pin = 3;  // MUX select (fsim/simulation.cpp:703)
      atomicAdd(indeg + dst, 1u);
      atomicMax(slot + (size_t)dst * 4 + (pin - 1), e + 1);
    }
  }
}

__global__ void k_line_keys(uint32_t W, const uint32_t* __restrict__ line_src, uint32_t* __restrict__ key,
                            uint32_t* __restrict__ id) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
    key[w] = line_src[w];
    id[w] = w;
  }
}

__global__ void k_gather_k(uint32_t W, const uint32_t* __restrict__ id, const uint32_t* __restrict__ line_k,
                           uint32_t* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W; i += gridDim.x * blockDim.x)
    out[i] = line_k[id[i]];
}

__global__ void k_scatter_rank(uint32_t W, const uint32_t* __restrict__ id, const uint32_t* __restrict__ r,
                               uint32_t* __restrict__ rank) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W; i += gridDim.x * blockDim.x)
    rank[id[i]] = r[i];
}

// Adjacency in insertion order: line w's sinks follow every earlier line of
// the same source (its rank).
__global__ void k_adj(uint32_t W, const uint32_t* __restrict__ a, const uint32_t* __restrict__ line_src,
                      const uint32_t* __restrict__ line_k, const uint32_t* __restrict__ line_off,
                      const uint32_t* __restrict__ line_rank, const uint32_t* __restrict__ adj_off,
                      uint32_t* __restrict__ adj) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
    const uint32_t k = line_k[w], off = line_off[w];
    const uint32_t base = adj_off[line_src[w]] + line_rank[w];
    for (uint32_t j = 0; j < k; ++j) adj[base + j] = a[off + 2 * j];
  }
}

__global__ void k_init_pis(uint32_t nPI, uint32_t* __restrict__ front, uint32_t* __restrict__ pos,
                           uint32_t* __restrict__ lev) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nPI; i += gridDim.x * blockDim.x) {
    front[i] = i;
    pos[i] = i;
    lev[i] = 0;
  }
}

// Wave step 1: every edge out of the wave records its FIFO key at the sink
// and takes one of the sink's pending inputs.
__global__ void k_wave_push(uint32_t n, uint32_t base, const uint32_t* __restrict__ front,
                            const uint32_t* __restrict__ adj_off, const uint32_t* __restrict__ adj,
                            unsigned long long* key, uint32_t* wait) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t u = front[i];
    const uint64_t hi = (uint64_t)(base + i) << 32;
    const uint32_t r0 = adj_off[u], r1 = adj_off[u + 1];
    for (uint32_t r = r0; r < r1; ++r) {
      const uint32_t v = adj[r];
      atomicMax(key + v, (unsigned long long)(hi | (r - r0)));
      atomicSub(wait + v, 1u);
    }
  }
}

// Wave step 2: per wave element, how many elements its edges append (their
// last input was this edge); POs are only counted as reached.
__global__ void k_wave_count(Dims d, uint32_t n, uint32_t base, const uint32_t* __restrict__ front,
                             const uint32_t* __restrict__ adj_off, const uint32_t* __restrict__ adj,
                             const unsigned long long* __restrict__ key, const uint32_t* __restrict__ wait,
                             uint32_t* __restrict__ cnt, Ctl* ctl) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t u = front[i];
    const uint64_t hi = (uint64_t)(base + i) << 32;
    const uint32_t r0 = adj_off[u], r1 = adj_off[u + 1];
    uint32_t c = 0;
    for (uint32_t r = r0; r < r1; ++r) {
      const uint32_t v = adj[r];
      if (wait[v] == 0 && key[v] == (hi | (r - r0))) {
        if (is_po(d, v))
          atomicAdd(&ctl->po_reached, 1u);
        else
          ++c;
      }
    }
    cnt[i] = c;
  }
}

// Wave step 3: the next wave in FIFO order, with positions and levels
// (fsim/simulation.cpp:882-893: 1 + the largest level over pin slots
// 1..count; an empty slot reads element 0).
__global__ void k_wave_emit(Dims d, uint32_t n, uint32_t base, uint32_t nbase,
                            const uint32_t* __restrict__ front, const uint32_t* __restrict__ adj_off,
                            const uint32_t* __restrict__ adj, const unsigned long long* __restrict__ key,
                            const uint32_t* __restrict__ wait, const uint32_t* __restrict__ cnt,
                            const uint32_t* __restrict__ offs, const uint32_t* __restrict__ indeg,
                            const uint32_t* __restrict__ slot, const uint32_t* __restrict__ esrc,
                            const uint8_t* __restrict__ types, uint32_t* __restrict__ next,
                            uint32_t* __restrict__ pos, uint32_t* lev, Ctl* ctl) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i == n - 1) ctl->next_n = offs[i] + cnt[i];
    const uint32_t u = front[i];
    const uint64_t hi = (uint64_t)(base + i) << 32;
    const uint32_t r0 = adj_off[u], r1 = adj_off[u + 1];
    uint32_t o = offs[i];
    for (uint32_t r = r0; r < r1; ++r) {
      const uint32_t v = adj[r];
      if (wait[v] != 0 || key[v] != (hi | (r - r0)) || is_po(d, v)) continue;
      next[o] = v;
      pos[v] = nbase + o;
      ++o;
      const uint32_t c = indeg[v];
      if (c > 4) {
        atomicOr(&ctl->err, kTooManyInputs);
        continue;
      }
      uint32_t lv = 0;
      for (uint32_t j = 0; j < c; ++j) {
        const uint32_t e = slot[(size_t)v * 4 + j];
        const uint32_t s = e ? esrc[e - 1] : 0u;
        lv = max(lv, lev[s] + 1);
      }
      lev[v] = lv;
      atomicMax(&ctl->max_level, lv);
      if (types[v - d.nPI - d.nPO] == G_MUX && c < 3) atomicOr(&ctl->err, kMuxInputs);
    }
  }
}

// Topological arrays: position of every element, types, levels, fanin counts.
__global__ void k_place(Dims d, const uint32_t* __restrict__ pos, const uint32_t* __restrict__ lev,
                        const uint32_t* __restrict__ indeg, const uint8_t* __restrict__ types,
                        unsigned long long* __restrict__ tpg, uint32_t* __restrict__ order,
                        uint8_t* __restrict__ type_t, uint32_t* __restrict__ level_t,
                        uint32_t* __restrict__ fcount, Ctl* ctl) {
  const uint32_t maxl = ctl->max_level;
  for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < d.N; f += gridDim.x * blockDim.x) {
    uint32_t t, lv;
    uint8_t ty;
    if (f < d.nPI) {
      t = pos[f];
      lv = 0;
      ty = G_PI;
    } else if (is_po(d, f)) {
      t = d.nPI + d.nG + (f - d.nPI);  // fsim/simulation.cpp:742-751
      lv = maxl + 1;
      ty = G_PO;
      if (indeg[f] > 4) atomicOr(&ctl->err, kTooManyInputs);
      if (indeg[f] == 0) atomicOr(&ctl->err, kNoInput);
    } else {
      t = pos[f];
      lv = lev[f];
      ty = types[f - d.nPI - d.nPO];
    }
    tpg[f] = t;
    order[t] = f;
    type_t[t] = ty;
    level_t[t] = lv;
    fcount[t] = f < d.nPI ? 0u : min(indeg[f], 4u);
  }
}

__global__ void k_fanin(Dims d, const uint32_t* __restrict__ order, const uint32_t* __restrict__ fcount,
                        const uint32_t* __restrict__ fi_off, const uint32_t* __restrict__ slot,
                        const uint32_t* __restrict__ esrc, const unsigned long long* __restrict__ tpg,
                        uint32_t* __restrict__ fi_idx, uint32_t* __restrict__ cons, uint8_t* __restrict__ fpin,
                        uint32_t* fo_cnt) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < d.N; t += gridDim.x * blockDim.x) {
    const uint32_t f = order[t], c = fcount[t], k0 = fi_off[t];
    for (uint32_t j = 0; j < c; ++j) {
      const uint32_t e = slot[(size_t)f * 4 + j];
      const uint32_t s = (uint32_t)tpg[e ? esrc[e - 1] : 0u];
      fi_idx[k0 + j] = s;
      cons[k0 + j] = t;
      fpin[k0 + j] = (uint8_t)j;
      atomicAdd(fo_cnt + s, 1u);
    }
  }
}

__global__ void k_sorted(uint32_t N, const uint32_t* __restrict__ level_t, Ctl* ctl) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x + 1; t < N; t += gridDim.x * blockDim.x)
    if (level_t[t] < level_t[t - 1]) ctl->unsorted = 1;
}

__global__ void k_fanout(uint32_t E, const uint32_t* __restrict__ val, const uint32_t* __restrict__ cons,
                         const uint8_t* __restrict__ fpin, uint32_t* __restrict__ fo_idx,
                         uint8_t* __restrict__ fo_pin) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < E; i += gridDim.x * blockDim.x) {
    const uint32_t k = val[i];
    fo_idx[i] = cons[k];
    fo_pin[i] = fpin[k];
  }
}

template <class T>
void zero(DevBuf& b, size_t count, cudaStream_t s) {
  b.ensure(count * sizeof(T));
  CK(cudaMemsetAsync(b.p, 0, count * sizeof(T), s));
}

template <class T>
void put(DevBuf& b, const T* src, size_t count, cudaStream_t s) {
  b.ensure(count * sizeof(T));
  if (count) CK(cudaMemcpyAsync(b.p, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
}

template <class T>
void get(std::vector<T>& v, const DevBuf& b, size_t count, cudaStream_t s) {
  v.resize(count);
  if (count) CK(cudaMemcpyAsync(v.data(), b.p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
}

// Exclusive sum of in[0, n) into out[0, n]; out[n] = total.
void exclusive_sum(LoaderDev& D, const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t s) {
  size_t bytes = 0;
  CK(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out + 1, n, s));
  D.temp.ensure(bytes);
  CK(cudaMemsetAsync(out, 0, sizeof(uint32_t), s));
  if (n) CK(cub::DeviceScan::InclusiveSum(D.temp.p, bytes, in, out + 1, n, s));
}

int bits_for(uint64_t max_value) {
  int b = 1;
  while (b < 32 && (max_value >> b)) ++b;
  return b;
}

}  // namespace

// Parallel tokenizer: every whitespace-separated token is a decimal number
// below 2^32.  Returns false on anything else.
static bool tokenize(const char* text, size_t len, int threads, std::unique_ptr<uint32_t[]>& out,
                     size_t& n_out) {
  const size_t T = (size_t)std::max(1, threads);
  std::vector<size_t> cut(T + 1);
  for (size_t i = 0; i <= T; ++i) {
    size_t b = len * i / T;
    while (b < len && b > 0 && !ws(text[b - 1]) && !ws(text[b])) ++b;  // never inside a token
    cut[i] = i == T ? len : b;
  }
  std::vector<size_t> count(T, 0);
  std::vector<uint8_t> ok(T, 1);
  auto run = [&](auto&& body) {
    std::vector<std::thread> ts;
    for (size_t i = 1; i < T; ++i) ts.emplace_back(body, i);
    body(0);
    for (auto& t : ts) t.join();
  };
  run([&](size_t i) {
    size_t c = 0;
    bool in = cut[i] > 0 && !ws(text[cut[i] - 1]);  // a token running into this chunk belongs to the one before
    for (size_t p = cut[i]; p < cut[i + 1]; ++p) {
      const bool w = ws(text[p]);
      if (!w && !in) ++c;
      in = !w;
    }
    count[i] = c;
  });
  std::vector<size_t> start(T + 1, 0);
  for (size_t i = 0; i < T; ++i) start[i + 1] = start[i] + count[i];
  if (start[T] >= (1ull << 32)) return false;
  n_out = start[T];
  out.reset(new uint32_t[n_out + 1]);
  run([&](size_t i) {
    const char* p = text + cut[i];
    const char* e = text + cut[i + 1];
    uint32_t* o = out.get() + start[i];
    while (true) {
      while (p < e && ws(*p)) ++p;
      if (p >= e) break;
      uint64_t v = 0;
      int nd = 0;
      while (p < e && (unsigned)(*p - '0') < 10u) {
        v = v * 10 + (uint64_t)(*p - '0');
        ++p;
        if (++nd > 10) {
          ok[i] = 0;
          return;
        }
      }
      if (nd == 0 || v > 0xFFFFFFFFull || (p < e && !ws(*p))) {
        ok[i] = 0;
        return;
      }
      *o++ = (uint32_t)v;
    }
  });
  for (size_t i = 0; i < T; ++i)
    if (!ok[i]) return false;
  return true;
}

bool parse_ckt_device(const char* text, size_t len, Netlist& nl, int device, cudaStream_t s, int threads,
                      LoadInfo& info) {
  const auto t0 = std::chrono::steady_clock::now();
  if (threads <= 0) {  // the hardware threads, at most 32, at least 1 MiB each
    threads = (int)std::min<unsigned>(32, std::max(1u, std::thread::hardware_concurrency()));
    threads = (int)std::max<size_t>(1, std::min<size_t>((size_t)threads, len / (1 << 20) + 1));
  }
  threads = (int)std::max<size_t>(1, std::min<size_t>((size_t)threads, len));
  info = LoadInfo{};
  info.threads = threads;
  std::unique_ptr<uint32_t[]> buf;
  size_t na = 0;
  if (!tokenize(text, len, threads, buf, na)) return false;
  const uint32_t* a = buf.get();

  // Structure (sequential: a line's length is in the line).
  if (na < 4) return false;
  const uint64_t nPI = a[0], nPO = a[1], nG = a[2], W = a[3];
  const uint64_t N64 = nPI + nPO + nG;
  if (nPI == 0 || N64 >= (1ull << 31) || W > len) return false;
  const uint32_t N = (uint32_t)N64;
  std::vector<uint32_t> line_src(W), line_k(W), line_off(W), line_eoff(W);
  uint64_t p = 4, E = 0;
  for (uint64_t w = 0; w < W; ++w) {
    if (p + 3 > na) return false;
    const uint32_t src = a[p], k = a[p + 2];
    if (src >= N || (src >= nPI && src < nPI + nPO)) return false;
    if (p + 3 + 2 * (uint64_t)k > na) return false;
    line_src[w] = src;
    line_k[w] = k;
    line_off[w] = (uint32_t)(p + 3);
    line_eoff[w] = (uint32_t)E;
    E += k;
    p += 3 + 2 * (uint64_t)k;
  }
  if (E >= (1ull << 31) || p + nG > na) return false;
  std::vector<uint8_t> types(nG);
  for (uint64_t i = 0; i < nG; ++i) {
    if (a[p + i] > 8) return false;
    types[i] = (uint8_t)a[p + i];
  }
  info.ms_tokenize = ms_since(t0);

  const auto t1 = std::chrono::steady_clock::now();
  CK(cudaSetDevice(device));
  LoaderDev D;
  const Dims d{N, (uint32_t)nPI, (uint32_t)nPO, (uint32_t)nG};
  const uint32_t Wn = (uint32_t)W, En = (uint32_t)E;
  put(D.a, a, na, s);
  put(D.line_src, line_src.data(), W, s);
  put(D.line_k, line_k.data(), W, s);
  put(D.line_off, line_off.data(), W, s);
  put(D.line_eoff, line_eoff.data(), W, s);
  put(D.types, types.data(), nG, s);
  zero<uint32_t>(D.indeg, N, s);
  zero<uint32_t>(D.slot, (size_t)N * 4, s);
  zero<uint32_t>(D.outdeg, N, s);
  zero<Ctl>(D.ctl, 1, s);
  D.esrc.ensure((size_t)En * 4);
  Ctl* ctl = D.ctl.as<Ctl>();
  if (Wn)
    k_edges<<<grid_for(Wn), kBlock, 0, s>>>(d, Wn, D.a.as<uint32_t>(), D.line_src.as<uint32_t>(),
                                            D.line_k.as<uint32_t>(), D.line_off.as<uint32_t>(),
                                            D.line_eoff.as<uint32_t>(), D.indeg.as<uint32_t>(),
                                            D.slot.as<uint32_t>(), D.esrc.as<uint32_t>(),
                                            D.outdeg.as<uint32_t>(), ctl);
  CK(cudaGetLastError());
  // Every sink must be in range before the adjacency and the waves index by it.
  Ctl hc{};
  CK(cudaMemcpyAsync(&hc, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (hc.err) return false;

  // Rank of each line among the lines of its source: a stable sort of the
  // lines by source, then a running sum of fanout counts per source.
  D.line_rank.ensure((size_t)Wn * 4 + 4);
  D.adj_off.ensure(((size_t)N + 1) * 4);
  exclusive_sum(D, D.outdeg.as<uint32_t>(), D.adj_off.as<uint32_t>(), N, s);
  if (Wn) {
    D.line_key.ensure((size_t)Wn * 4);
    D.line_key2.ensure((size_t)Wn * 4);
    D.line_id.ensure((size_t)Wn * 4);
    D.line_id2.ensure((size_t)Wn * 4);
    D.line_ksorted.ensure((size_t)Wn * 4);
    D.line_rsorted.ensure((size_t)Wn * 4);
    k_line_keys<<<grid_for(Wn), kBlock, 0, s>>>(Wn, D.line_src.as<uint32_t>(), D.line_key.as<uint32_t>(),
                                                D.line_id.as<uint32_t>());
    size_t bytes = 0;
    const int nb = bits_for(N);
    CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, D.line_key.as<uint32_t>(), D.line_key2.as<uint32_t>(),
                                       D.line_id.as<uint32_t>(), D.line_id2.as<uint32_t>(), Wn, 0, nb, s));
    D.temp.ensure(bytes);
    CK(cub::DeviceRadixSort::SortPairs(D.temp.p, bytes, D.line_key.as<uint32_t>(), D.line_key2.as<uint32_t>(),
                                       D.line_id.as<uint32_t>(), D.line_id2.as<uint32_t>(), Wn, 0, nb, s));
    k_gather_k<<<grid_for(Wn), kBlock, 0, s>>>(Wn, D.line_id2.as<uint32_t>(), D.line_k.as<uint32_t>(),
                                               D.line_ksorted.as<uint32_t>());
    bytes = 0;
    CK(cub::DeviceScan::ExclusiveSumByKey(nullptr, bytes, D.line_key2.as<uint32_t>(),
                                          D.line_ksorted.as<uint32_t>(), D.line_rsorted.as<uint32_t>(), Wn,
                                          cub::Equality(), s));
    D.temp.ensure(bytes);
    CK(cub::DeviceScan::ExclusiveSumByKey(D.temp.p, bytes, D.line_key2.as<uint32_t>(),
                                          D.line_ksorted.as<uint32_t>(), D.line_rsorted.as<uint32_t>(), Wn,
                                          cub::Equality(), s));
    k_scatter_rank<<<grid_for(Wn), kBlock, 0, s>>>(Wn, D.line_id2.as<uint32_t>(), D.line_rsorted.as<uint32_t>(),
                                                   D.line_rank.as<uint32_t>());
    D.adj.ensure((size_t)En * 4 + 4);
    k_adj<<<grid_for(Wn), kBlock, 0, s>>>(Wn, D.a.as<uint32_t>(), D.line_src.as<uint32_t>(),
                                          D.line_k.as<uint32_t>(), D.line_off.as<uint32_t>(),
                                          D.line_rank.as<uint32_t>(), D.adj_off.as<uint32_t>(),
                                          D.adj.as<uint32_t>());
    CK(cudaGetLastError());
  }
  D.a.release();

  // Waves.
  zero<unsigned long long>(D.key, N, s);
  D.pos.ensure((size_t)N * 4);
  CK(cudaMemsetAsync(D.pos.p, 0xFF, (size_t)N * 4, s));
  D.lev.ensure((size_t)N * 4);
  D.wait.ensure((size_t)N * 4);
  CK(cudaMemcpyAsync(D.wait.p, D.indeg.p, (size_t)N * 4, cudaMemcpyDeviceToDevice, s));
  D.front[0].ensure((size_t)N * 4);
  D.front[1].ensure((size_t)N * 4);
  D.cnt.ensure((size_t)N * 4);
  D.offs.ensure(((size_t)N + 1) * 4);
  {
    size_t bytes = 0;
    CK(cub::DeviceScan::InclusiveSum(nullptr, bytes, D.cnt.as<uint32_t>(), D.offs.as<uint32_t>(), N, s));
    D.temp.ensure(bytes);
  }
  k_init_pis<<<grid_for(nPI), kBlock, 0, s>>>((uint32_t)nPI, D.front[0].as<uint32_t>(), D.pos.as<uint32_t>(),
                                               D.lev.as<uint32_t>());
  CK(cudaGetLastError());
  uint32_t n = (uint32_t)nPI, base = 0, cur = 0, waves = 0;
  while (n) {
    const uint32_t nbase = base + n;
    uint32_t* fr = D.front[cur].as<uint32_t>();
    k_wave_push<<<grid_for(n), kBlock, 0, s>>>(n, base, fr, D.adj_off.as<uint32_t>(), D.adj.as<uint32_t>(),
                                               D.key.as<unsigned long long>(), D.wait.as<uint32_t>());
    k_wave_count<<<grid_for(n), kBlock, 0, s>>>(d, n, base, fr, D.adj_off.as<uint32_t>(), D.adj.as<uint32_t>(),
                                                D.key.as<unsigned long long>(), D.wait.as<uint32_t>(),
                                                D.cnt.as<uint32_t>(), ctl);
    exclusive_sum(D, D.cnt.as<uint32_t>(), D.offs.as<uint32_t>(), n, s);
    k_wave_emit<<<grid_for(n), kBlock, 0, s>>>(
        d, n, base, nbase, fr, D.adj_off.as<uint32_t>(), D.adj.as<uint32_t>(), D.key.as<unsigned long long>(),
        D.wait.as<uint32_t>(), D.cnt.as<uint32_t>(), D.offs.as<uint32_t>(), D.indeg.as<uint32_t>(),
        D.slot.as<uint32_t>(), D.esrc.as<uint32_t>(), D.types.as<uint8_t>(), D.front[cur ^ 1].as<uint32_t>(),
        D.pos.as<uint32_t>(), D.lev.as<uint32_t>(), ctl);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&hc, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ++waves;
    if (hc.err) return false;
    base = nbase;
    n = hc.next_n;
    cur ^= 1;
  }
  info.waves = waves;
  if (base != nPI + nG || hc.po_reached != nPO) return false;  // unreachable elements

  // Topological arrays.
  D.tpg.ensure((size_t)N * 8);
  D.order.ensure((size_t)N * 4);
  D.type_t.ensure(N);
  D.level_t.ensure((size_t)N * 4);
  D.fcount.ensure((size_t)N * 4);
  k_place<<<grid_for(N), kBlock, 0, s>>>(d, D.pos.as<uint32_t>(), D.lev.as<uint32_t>(), D.indeg.as<uint32_t>(),
                                         D.types.as<uint8_t>(), D.tpg.as<unsigned long long>(),
                                         D.order.as<uint32_t>(), D.type_t.as<uint8_t>(),
                                         D.level_t.as<uint32_t>(), D.fcount.as<uint32_t>(), ctl);
  D.fi_off.ensure(((size_t)N + 1) * 4);
  exclusive_sum(D, D.fcount.as<uint32_t>(), D.fi_off.as<uint32_t>(), N, s);
  D.fi_idx.ensure((size_t)En * 4 + 4);
  D.cons.ensure((size_t)En * 4 + 4);
  D.fpin.ensure((size_t)En + 4);
  zero<uint32_t>(D.fo_cnt, N, s);
  k_fanin<<<grid_for(N), kBlock, 0, s>>>(d, D.order.as<uint32_t>(), D.fcount.as<uint32_t>(),
                                          D.fi_off.as<uint32_t>(), D.slot.as<uint32_t>(), D.esrc.as<uint32_t>(),
                                          D.tpg.as<unsigned long long>(), D.fi_idx.as<uint32_t>(),
                                          D.cons.as<uint32_t>(), D.fpin.as<uint8_t>(), D.fo_cnt.as<uint32_t>());
  k_sorted<<<grid_for(N), kBlock, 0, s>>>(N, D.level_t.as<uint32_t>(), ctl);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(&hc, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (hc.err || hc.unsorted) return false;

  // Fanout CSR: fanin entries stably sorted by source keep consumers
  // ascending and, per consumer, pins ascending.
  D.fo_off.ensure(((size_t)N + 1) * 4);
  exclusive_sum(D, D.fo_cnt.as<uint32_t>(), D.fo_off.as<uint32_t>(), N, s);
  D.fo_key.ensure((size_t)En * 4 + 4);
  D.fo_val.ensure((size_t)En * 4 + 4);
  D.fo_val2.ensure((size_t)En * 4 + 4);
  D.fo_idx.ensure((size_t)En * 4 + 4);
  D.fo_pin.ensure((size_t)En + 4);
  if (En) {
    k_line_keys<<<grid_for(En), kBlock, 0, s>>>(En, D.fi_idx.as<uint32_t>(), D.fo_key.as<uint32_t>(),
                                                D.fo_val.as<uint32_t>());
    D.fo_key2.ensure((size_t)En * 4 + 4);
    size_t bytes = 0;
    const int nb = bits_for(N);
    CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, D.fo_key.as<uint32_t>(), D.fo_key2.as<uint32_t>(),
                                       D.fo_val.as<uint32_t>(), D.fo_val2.as<uint32_t>(), En, 0, nb, s));
    D.temp.ensure(bytes);
    CK(cub::DeviceRadixSort::SortPairs(D.temp.p, bytes, D.fo_key.as<uint32_t>(), D.fo_key2.as<uint32_t>(),
                                       D.fo_val.as<uint32_t>(), D.fo_val2.as<uint32_t>(), En, 0, nb, s));
    k_fanout<<<grid_for(En), kBlock, 0, s>>>(En, D.fo_val2.as<uint32_t>(), D.cons.as<uint32_t>(),
                                             D.fpin.as<uint8_t>(), D.fo_idx.as<uint32_t>(),
                                             D.fo_pin.as<uint8_t>());
    CK(cudaGetLastError());
  }

  Netlist out;
  out.n_pi = nPI;
  out.n_po = nPO;
  out.n_gates = nG;
  out.n_wires = W;
  out.N = N;
  std::vector<unsigned long long> tpg;
  get(tpg, D.tpg, N, s);
  get(out.type, D.type_t, N, s);
  get(out.level, D.level_t, N, s);
  get(out.fi_off, D.fi_off, (size_t)N + 1, s);
  get(out.fi_idx, D.fi_idx, En, s);
  get(out.fo_off, D.fo_off, (size_t)N + 1, s);
  get(out.fo_idx, D.fo_idx, En, s);
  get(out.fo_pin, D.fo_pin, En, s);
  CK(cudaStreamSynchronize(s));
  out.tpg.assign(tpg.begin(), tpg.end());
  out.n_levels = hc.max_level + 2;
  out.per_level.assign(out.n_levels, 0);
  for (uint32_t t = 0; t < N; ++t) out.per_level[out.level[t]]++;
  out.level_off.assign(out.n_levels + 1, 0);
  for (uint32_t l = 0; l < out.n_levels; ++l) out.level_off[l + 1] = out.level_off[l] + (uint32_t)out.per_level[l];
  nl = std::move(out);
  info.on_device = true;
  info.ms_device = ms_since(t1);
  info.ms_total = ms_since(t0);
  return true;
}

}  // namespace fsimb
