/*
 * CPU oracle -- TEST INFRASTRUCTURE (see fsim_oracle.h).  A plain-C
 * restatement of fsim/simulation.cpp; each step cites the lines it follows.
 */
#define _GNU_SOURCE
#include "fsim_oracle.h"

#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { T_INV = 0, T_AND, T_OR, T_XOR, T_NAND, T_NOR, T_XNOR, T_MUX, T_CLKBUF, T_PI, T_PO };

struct or_netlist {
  uint64_t n_pi, n_po, n_gates, n_wires, N;
  uint8_t* type;      /* [N] by topological index */
  uint64_t* fi_off;   /* [N+1] */
  uint64_t* fi_idx;   /* fanins, pin order */
  uint64_t* fo_off;   /* [N+1] */
  uint64_t* fo_idx;
  uint64_t* tpg;      /* file id -> topological index */
  uint64_t* level;    /* [N] */
  uint64_t n_levels;
  uint64_t* per_level;
  uint64_t po_begin;  /* first PO topological index */
};

/* ---- tokenizer (std::istream >> size_t) ---- */
typedef struct {
  const char* p;
  const char* e;
  int bad;
} tok_t;

static int tok_u64(tok_t* t, uint64_t* v) {
  while (t->p < t->e && (*t->p == ' ' || *t->p == '\n' || *t->p == '\t' || *t->p == '\r'))
    t->p++;
  if (t->p >= t->e || *t->p < '0' || *t->p > '9') {
    t->bad = 1;
    return 0;
  }
  uint64_t x = 0;
  while (t->p < t->e && *t->p >= '0' && *t->p <= '9') x = x * 10 + (uint64_t)(*t->p++ - '0');
  *v = x;
  return 1;
}

#define FAIL(...)                           \
  do {                                      \
    if (err) snprintf(err, errlen, __VA_ARGS__); \
    goto fail;                              \
  } while (0)

/* fsim/simulation.cpp:37-41, 664-941 */
or_netlist* or_parse_ckt(const char* text, size_t len, char* err, size_t errlen) {
  tok_t t = {text, text + len, 0};
  or_netlist* nl = calloc(1, sizeof *nl);
  uint64_t* table = NULL; /* gate_input_order_table: 5 slots per element */
  uint64_t *adj_cnt = NULL, *adj_off = NULL, *adj = NULL, *indeg = NULL, *order = NULL;
  uint64_t *e_src = NULL, *e_dst = NULL;
  uint8_t* ftype = NULL;
  if (!tok_u64(&t, &nl->n_pi) || !tok_u64(&t, &nl->n_po) || !tok_u64(&t, &nl->n_gates) ||
      !tok_u64(&t, &nl->n_wires))
    FAIL("ckt header");
  const uint64_t N = nl->n_pi + nl->n_po + nl->n_gates;
  nl->N = N;
  if (nl->n_pi == 0 || N > (1ull << 31)) FAIL("ckt size");
  table = calloc(N * 5, sizeof(uint64_t));
  indeg = calloc(N, sizeof(uint64_t));
  size_t ecap = 16, ne = 0;
  e_src = malloc(ecap * sizeof(uint64_t));
  e_dst = malloc(ecap * sizeof(uint64_t));
  /* wires: adjacency, indegree and pin table (fsim/simulation.cpp:684-711) */
  for (uint64_t i = 0; i < nl->n_wires; i++) {
    uint64_t g0, pinY, k;
    if (!tok_u64(&t, &g0) || !tok_u64(&t, &pinY) || !tok_u64(&t, &k)) FAIL("ckt wire line");
    if (g0 >= N || (g0 >= nl->n_pi && g0 < nl->n_pi + nl->n_po)) FAIL("ckt wire source");
    for (uint64_t j = 0; j < k; j++) {
      uint64_t dst, pin;
      if (!tok_u64(&t, &dst) || !tok_u64(&t, &pin)) FAIL("ckt wire sink");
      if (dst >= N || dst < nl->n_pi || pin < 1 || pin > 5) FAIL("ckt wire sink range");
      pin = (pin == 5) ? 3 : pin; /* MUX select (fsim/simulation.cpp:703) */
      if (table[dst * 5] >= 4) FAIL("ckt fan-in above 4");
      table[dst * 5 + pin] = g0;
      table[dst * 5]++;
      indeg[dst]++;
      if (ne == ecap) {
        ecap *= 2;
        e_src = realloc(e_src, ecap * sizeof(uint64_t));
        e_dst = realloc(e_dst, ecap * sizeof(uint64_t));
      }
      e_src[ne] = g0;
      e_dst[ne] = dst;
      ne++;
    }
  }
  adj_cnt = calloc(N + 1, sizeof(uint64_t));
  adj_off = calloc(N + 1, sizeof(uint64_t));
  adj = malloc((ne + 1) * sizeof(uint64_t));
  for (size_t k = 0; k < ne; k++) adj_cnt[e_src[k]]++;
  for (uint64_t i = 0; i < N; i++) adj_off[i + 1] = adj_off[i] + adj_cnt[i];
  memset(adj_cnt, 0, (N + 1) * sizeof(uint64_t));
  for (size_t k = 0; k < ne; k++) adj[adj_off[e_src[k]] + adj_cnt[e_src[k]]++] = e_dst[k];

  /* Kahn's algorithm, FIFO seeded with the PIs (fsim/simulation.cpp:718-738) */
  order = malloc((N + 1) * sizeof(uint64_t));
  uint64_t head = 0, tail = 0;
  for (uint64_t i = 0; i < nl->n_pi; i++) order[tail++] = i;
  while (head < tail) {
    uint64_t u = order[head++];
    for (uint64_t k = adj_off[u]; k < adj_off[u + 1]; k++) {
      uint64_t v = adj[k];
      if (--indeg[v] == 0) {
        if (tail >= N) FAIL("ckt order overflow");
        order[tail++] = v;
      }
    }
  }
  /* drop POs, then append them in id order (fsim/simulation.cpp:742-751) */
  uint64_t n = 0;
  for (uint64_t i = 0; i < tail; i++) {
    uint64_t x = order[i];
    if (!(x >= nl->n_pi && x < nl->n_pi + nl->n_po)) order[n++] = x;
  }
  for (uint64_t i = 0; i < nl->n_po; i++) order[n++] = nl->n_pi + i;
  if (n != N) FAIL("ckt: %llu element(s) unreachable", (unsigned long long)(N - n));

  /* types (fsim/simulation.cpp:760-772) */
  ftype = malloc(N);
  for (uint64_t i = 0; i < N; i++) {
    if (i < nl->n_pi)
      ftype[i] = T_PI;
    else if (i < nl->n_pi + nl->n_po)
      ftype[i] = T_PO;
    else {
      uint64_t ty;
      if (!tok_u64(&t, &ty) || ty > 8) FAIL("ckt gate type");
      ftype[i] = (uint8_t)ty;
    }
  }
  /* id -> topological index (fsim/simulation.cpp:781-784) */
  nl->tpg = malloc(N * sizeof(uint64_t));
  for (uint64_t i = 0; i < N; i++) nl->tpg[order[i]] = i;
  nl->type = malloc(N);
  nl->fi_off = calloc(N + 1, sizeof(uint64_t));
  nl->fi_idx = malloc((4 * N + 1) * sizeof(uint64_t));
  /* fanins from pin slots 1..count (fsim/simulation.cpp:851-877) */
  uint64_t m = 0;
  for (uint64_t ti = 0; ti < N; ti++) {
    uint64_t f = order[ti];
    nl->type[ti] = ftype[f];
    nl->fi_off[ti] = m;
    if (ti >= nl->n_pi) {
      uint64_t cnt = table[f * 5];
      if (cnt == 0) FAIL("ckt: element without input");
      if (ftype[f] == T_MUX && cnt < 3) FAIL("ckt: MUX with fewer than 3 inputs");
      for (uint64_t j = 1; j <= cnt; j++) nl->fi_idx[m++] = nl->tpg[table[f * 5 + j]];
    }
  }
  nl->fi_off[N] = m;
  /* levels (fsim/simulation.cpp:882-916) */
  nl->level = calloc(N, sizeof(uint64_t));
  uint64_t maxl = 0;
  for (uint64_t ti = nl->n_pi; ti < nl->n_pi + nl->n_gates; ti++) {
    uint64_t lv = nl->level[nl->fi_idx[nl->fi_off[ti]]] + 1;
    for (uint64_t k = nl->fi_off[ti] + 1; k < nl->fi_off[ti + 1]; k++)
      if (nl->level[nl->fi_idx[k]] + 1 > lv) lv = nl->level[nl->fi_idx[k]] + 1;
    nl->level[ti] = lv;
    if (lv > maxl) maxl = lv;
  }
  for (uint64_t ti = nl->n_pi + nl->n_gates; ti < N; ti++) nl->level[ti] = maxl + 1;
  nl->n_levels = maxl + 2;
  nl->per_level = calloc(nl->n_levels, sizeof(uint64_t));
  for (uint64_t ti = 0; ti < N; ti++) nl->per_level[nl->level[ti]]++;
  nl->po_begin = nl->n_pi + nl->n_gates;
  /* fanout lists, consumers ascending */
  nl->fo_off = calloc(N + 1, sizeof(uint64_t));
  nl->fo_idx = malloc((m + 1) * sizeof(uint64_t));
  for (uint64_t k = 0; k < m; k++) nl->fo_off[nl->fi_idx[k] + 1]++;
  for (uint64_t i = 0; i < N; i++) nl->fo_off[i + 1] += nl->fo_off[i];
  uint64_t* fill = malloc((N + 1) * sizeof(uint64_t));
  memcpy(fill, nl->fo_off, (N + 1) * sizeof(uint64_t));
  for (uint64_t ti = 0; ti < N; ti++)
    for (uint64_t k = nl->fi_off[ti]; k < nl->fi_off[ti + 1]; k++) nl->fo_idx[fill[nl->fi_idx[k]]++] = ti;
  free(fill);
  free(table);
  free(adj_cnt);
  free(adj_off);
  free(adj);
  free(indeg);
  free(order);
  free(e_src);
  free(e_dst);
  free(ftype);
  return nl;
fail:
  free(table);
  free(adj_cnt);
  free(adj_off);
  free(adj);
  free(indeg);
  free(order);
  free(e_src);
  free(e_dst);
  free(ftype);
  or_free(nl);
  return NULL;
}

void or_free(or_netlist* nl) {
  if (!nl) return;
  free(nl->type);
  free(nl->fi_off);
  free(nl->fi_idx);
  free(nl->fo_off);
  free(nl->fo_idx);
  free(nl->tpg);
  free(nl->level);
  free(nl->per_level);
  free(nl);
}

uint64_t or_num_elements(const or_netlist* nl) { return nl->N; }
uint64_t or_num_pis(const or_netlist* nl) { return nl->n_pi; }
uint64_t or_num_pos(const or_netlist* nl) { return nl->n_po; }
uint64_t or_num_gates(const or_netlist* nl) { return nl->n_gates; }
uint64_t or_num_levels(const or_netlist* nl) { return nl->n_levels; }
void or_tpg(const or_netlist* nl, uint64_t* out) { memcpy(out, nl->tpg, nl->N * 8); }
void or_levels(const or_netlist* nl, uint64_t* out) { memcpy(out, nl->level, nl->N * 8); }
void or_per_level(const or_netlist* nl, uint64_t* out) { memcpy(out, nl->per_level, nl->n_levels * 8); }
void or_types(const or_netlist* nl, uint8_t* out) { memcpy(out, nl->type, nl->N); }

/* fsim/simulation.cpp:943-959 (plus the extended pin column) */
int64_t or_parse_flst(const or_netlist* nl, const char* text, size_t len, or_fault* out,
                      size_t cap, char* err, size_t errlen) {
  tok_t t = {text, text + len, 0};
  int pins = 0;
  while (t.p < t.e && (*t.p == ' ' || *t.p == '\n' || *t.p == '\t' || *t.p == '\r')) t.p++;
  if (t.e - t.p >= 5 && memcmp(t.p, "@pins", 5) == 0) {
    pins = 1;
    t.p += 5;
  }
  uint64_t F;
  if (!tok_u64(&t, &F)) FAIL("flst count");
  if (F > cap) FAIL("flst capacity");
  for (uint64_t i = 0; i < F; i++) {
    uint64_t id, v, pin = 0;
    if (!tok_u64(&t, &id) || !tok_u64(&t, &v) || (pins && !tok_u64(&t, &pin))) FAIL("flst line");
    if (id >= nl->N) FAIL("flst site");
    out[i].site = nl->tpg[id];
    out[i].value = v ? 1 : 0;
    out[i].pin = (uint32_t)pin;
    if (pin > nl->fi_off[out[i].site + 1] - nl->fi_off[out[i].site]) FAIL("flst pin");
  }
  return (int64_t)F;
fail:
  return -1;
}

/* fsim/simulation.cpp:961-976; rows kept in file order (the identity
 * whenever ceil(P/64) <= nPI, the only case the reference defines). */
int64_t or_parse_ptn(const or_netlist* nl, const char* text, size_t len, uint64_t* out,
                     size_t cap, char* err, size_t errlen) {
  tok_t t = {text, text + len, 0};
  uint64_t P;
  if (!tok_u64(&t, &P)) FAIL("ptn count");
  uint64_t W = (P + 63) / 64;
  if (W * nl->n_pi > cap) FAIL("ptn capacity");
  for (uint64_t i = 0; i < W * nl->n_pi; i++)
    if (!tok_u64(&t, &out[i])) FAIL("ptn word");
  return (int64_t)P;
fail:
  return -1;
}

/* Gate functions (fsim/simulation.cpp:979-1077).  MUX keeps the reference's
 * logical not of the select word (fsim/simulation.cpp:1056). */
static inline uint64_t eval_gate(uint8_t ty, const uint64_t* in, uint64_t n) {
  uint64_t r = in[0];
  switch (ty) {
    case T_INV: return ~r;
    case T_AND:
      for (uint64_t i = 1; i < n; i++) r &= in[i];
      return r;
    case T_OR:
      for (uint64_t i = 1; i < n; i++) r |= in[i];
      return r;
    case T_XOR:
      for (uint64_t i = 1; i < n; i++) r ^= in[i];
      return r;
    case T_NAND:
      for (uint64_t i = 1; i < n; i++) r &= in[i];
      return ~r;
    case T_NOR:
      for (uint64_t i = 1; i < n; i++) r |= in[i];
      return ~r;
    case T_XNOR:
      for (uint64_t i = 1; i < n; i++) r ^= in[i];
      return ~r;
    case T_MUX: return (in[2] & in[1]) | (in[0] & (uint64_t)(!in[2]));
    case T_CLKBUF: return r;
    case T_PO: return r;
    default: return r;
  }
}

/* bits in round rd (fsim/simulation.cpp:115-118) */
static inline uint64_t round_bits(uint64_t P, uint64_t rd) {
  return (P / (64 * (rd + 1))) ? 64 : (P % 64);
}
/* _shift_to_correct_answer (fsim/simulation.cpp:94-102) as a mask */
static inline uint64_t bits_mask(uint64_t bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1); }

static void good_raw(const or_netlist* nl, const uint64_t* words, uint64_t rd, uint64_t* g) {
  for (uint64_t i = 0; i < nl->N; i++) {
    if (nl->type[i] == T_PI) {
      g[i] = words[rd * nl->n_pi + i]; /* _apply_PI: pattern word of PI i */
    } else {
      uint64_t in[4];
      uint64_t n = nl->fi_off[i + 1] - nl->fi_off[i];
      for (uint64_t k = 0; k < n; k++) in[k] = g[nl->fi_idx[nl->fi_off[i] + k]];
      g[i] = eval_gate(nl->type[i], in, n);
    }
  }
}

void or_good_values(const or_netlist* nl, const uint64_t* words, uint64_t P, uint64_t rd,
                    uint64_t* out) {
  good_raw(nl, words, rd, out);
  uint64_t m = bits_mask(round_bits(P, rd));
  for (uint64_t i = 0; i < nl->N; i++) out[i] &= m;
}

void or_results_init(or_result* res, size_t n) {
  for (size_t i = 0; i < n; i++) {
    memset(&res[i], 0, sizeof res[i]);
    res[i].first = -1;
  }
}

/* Fold one round's PO difference word into a fault's result. */
static void accumulate(or_result* r, uint64_t diff, uint64_t bits, uint64_t rd, uint64_t last_rd) {
  if (diff) {
    r->detected = 1;
    r->count += (uint64_t)__builtin_popcountll(diff);
    /* lowest pattern index = highest set bit: rd*64 + bits-1-b */
    int64_t b = 63 - __builtin_clzll(diff);
    int64_t idx = (int64_t)(rd * 64 + bits - 1) - b;
    if (r->first < 0 || idx < r->first) r->first = idx;
  }
  if (rd == last_rd) {
    r->ref_flag = diff != 0;
    r->ref_rd = rd;
  }
}

typedef struct {
  const or_netlist* nl;
  const or_fault* faults;
  uint64_t f0, f1;
  const uint64_t* words;
  uint64_t P, rd0, rd1;
  int mode;
  or_result* res; /* indexed by f - base */
  uint64_t base;
} job_t;

/* Full re-simulation per fault: _run_bad_case (fsim/simulation.cpp:186-228)
 * with the stuck value forced at the site; a pin fault forces one input. */
static void run_naive(const job_t* j) {
  const or_netlist* nl = j->nl;
  const uint64_t N = nl->N;
  uint64_t* g = malloc(N * 8);
  uint64_t* b = malloc(N * 8);
  const uint64_t W = (j->P + 63) / 64;
  for (uint64_t rd = j->rd0; rd < j->rd1; rd++) {
    const uint64_t bits = round_bits(j->P, rd), mask = bits_mask(bits);
    good_raw(nl, j->words, rd, g);
    for (uint64_t fi = j->f0; fi < j->f1; fi++) {
      const or_fault* f = &j->faults[fi];
      const uint64_t sv = f->value ? ~0ull : 0ull;
      for (uint64_t i = 0; i < N; i++) {
        if (i == f->site && f->pin == 0) {
          b[i] = sv;
          continue;
        }
        if (nl->type[i] == T_PI) {
          b[i] = j->words[rd * nl->n_pi + i];
          continue;
        }
        uint64_t in[4];
        uint64_t n = nl->fi_off[i + 1] - nl->fi_off[i];
        for (uint64_t k = 0; k < n; k++) in[k] = b[nl->fi_idx[nl->fi_off[i] + k]];
        if (i == f->site) in[f->pin - 1] = sv;
        b[i] = eval_gate(nl->type[i], in, n);
      }
      /* masked PO compare (fsim/simulation.cpp:134-140) */
      uint64_t diff = 0;
      for (uint64_t i = nl->po_begin; i < N; i++) diff |= (g[i] ^ b[i]) & mask;
      accumulate(&j->res[fi - j->base], diff, bits, rd, W - 1);
    }
  }
  free(g);
  free(b);
}

/* Same results, propagating only through the fault's fanout cone: pending
 * elements are bits of a bitmap scanned upward from the fault site.  Every
 * consumer has a larger topological index than its fanins, so one forward
 * scan visits the pending elements in topological order. */
static void run_event(const job_t* j) {
  const or_netlist* nl = j->nl;
  const uint64_t N = nl->N;
  const uint64_t NW = (N + 63) / 64;
  uint64_t* g = malloc(N * 8);
  uint64_t* b = malloc(N * 8);
  uint32_t* stamp = calloc(N, sizeof(uint32_t)); /* b[i] valid for this fault */
  uint64_t* pend = calloc(NW, sizeof(uint64_t));
  uint32_t epoch = 0;
  const uint64_t W = (j->P + 63) / 64;
  for (uint64_t rd = j->rd0; rd < j->rd1; rd++) {
    const uint64_t bits = round_bits(j->P, rd), mask = bits_mask(bits);
    good_raw(nl, j->words, rd, g);
    for (uint64_t fi = j->f0; fi < j->f1; fi++) {
      const or_fault* f = &j->faults[fi];
      const uint64_t sv = f->value ? ~0ull : 0ull;
      epoch++;
      pend[f->site >> 6] |= 1ull << (f->site & 63);
      uint64_t npend = 1;
      uint64_t diff = 0;
      for (uint64_t w = f->site >> 6; w < NW && npend; w++) {
        while (pend[w]) {
          const uint64_t i = w * 64 + (uint64_t)__builtin_ctzll(pend[w]);
          pend[w] &= pend[w] - 1;
          npend--;
          uint64_t v;
          if (i == f->site && f->pin == 0) {
            v = sv;
          } else {
            uint64_t in[4];
            uint64_t n = nl->fi_off[i + 1] - nl->fi_off[i];
            for (uint64_t k = 0; k < n; k++) {
              uint64_t d = nl->fi_idx[nl->fi_off[i] + k];
              in[k] = (stamp[d] == epoch) ? b[d] : g[d];
            }
            if (i == f->site) in[f->pin - 1] = sv;
            v = eval_gate(nl->type[i], in, n);
          }
          if (v == g[i]) continue; /* no difference leaves this element */
          b[i] = v;
          stamp[i] = epoch;
          if (i >= nl->po_begin) diff |= (g[i] ^ v) & mask;
          for (uint64_t k = nl->fo_off[i]; k < nl->fo_off[i + 1]; k++) {
            const uint64_t c = nl->fo_idx[k];
            const uint64_t m = 1ull << (c & 63);
            if (!(pend[c >> 6] & m)) {
              pend[c >> 6] |= m;
              npend++;
            }
          }
        }
      }
      accumulate(&j->res[fi - j->base], diff, bits, rd, W - 1);
    }
  }
  free(g);
  free(b);
  free(stamp);
  free(pend);
}

/* Gate functions over nr words at once (the same functions as eval_gate,
 * word by word). */
static void eval_vec(uint8_t ty, const uint64_t* const* in, uint64_t n, uint64_t* v, uint64_t nr) {
  uint64_t r, k;
  switch (ty) {
    case T_INV:
      for (r = 0; r < nr; r++) v[r] = ~in[0][r];
      return;
    case T_AND:
    case T_NAND:
      for (r = 0; r < nr; r++) {
        uint64_t x = in[0][r];
        for (k = 1; k < n; k++) x &= in[k][r];
        v[r] = ty == T_NAND ? ~x : x;
      }
      return;
    case T_OR:
    case T_NOR:
      for (r = 0; r < nr; r++) {
        uint64_t x = in[0][r];
        for (k = 1; k < n; k++) x |= in[k][r];
        v[r] = ty == T_NOR ? ~x : x;
      }
      return;
    case T_XOR:
    case T_XNOR:
      for (r = 0; r < nr; r++) {
        uint64_t x = in[0][r];
        for (k = 1; k < n; k++) x ^= in[k][r];
        v[r] = ty == T_XNOR ? ~x : x;
      }
      return;
    case T_MUX:
      for (r = 0; r < nr; r++) v[r] = (in[2][r] & in[1][r]) | (in[0][r] & (uint64_t)(!in[2][r]));
      return;
    default: /* CLKBUF, PO */
      for (r = 0; r < nr; r++) v[r] = in[0][r];
      return;
  }
}

/* The event-driven propagation of run_event for a chunk of up to R rounds
 * at once: an element is evaluated for every round of the chunk when any
 * of its fanins differs in any round, and the per-round PO differences are
 * folded into the results one round at a time.  Same results as modes 0
 * and 1; the chunk turns one random access per element into R words. */
static void run_event_chunked(const job_t* j) {
  const or_netlist* nl = j->nl;
  const uint64_t N = nl->N;
  const uint64_t NW = (N + 63) / 64;
  uint64_t R = (64ull << 20) / (N * 8 + 1); /* about 64 MB of faulty words per thread */
  if (R > 64) R = 64;
  if (R < 4) R = 4;
  uint64_t* g = malloc(N * R * 8);
  uint64_t* b = malloc(N * R * 8);
  uint32_t* stamp = calloc(N, sizeof(uint32_t));
  uint64_t* pend = calloc(NW, sizeof(uint64_t));
  uint64_t* v = malloc(R * 8);
  uint64_t* diff = malloc(R * 8);
  uint64_t* mask = malloc(R * 8);
  uint64_t* bitsv = malloc(R * 8);
  uint64_t* svv = malloc(R * 8);
  uint32_t epoch = 0;
  const uint64_t W = (j->P + 63) / 64;
  for (uint64_t c0 = j->rd0; c0 < j->rd1; c0 += R) {
    const uint64_t nr = (j->rd1 - c0 < R) ? j->rd1 - c0 : R;
    for (uint64_t r = 0; r < nr; r++) {
      bitsv[r] = round_bits(j->P, c0 + r);
      mask[r] = bits_mask(bitsv[r]);
    }
    /* good machine of the chunk, element-major [i][r] */
    for (uint64_t i = 0; i < N; i++) {
      uint64_t* gi = g + i * R;
      if (nl->type[i] == T_PI) {
        for (uint64_t r = 0; r < nr; r++) gi[r] = j->words[(c0 + r) * nl->n_pi + i];
      } else {
        const uint64_t* in[4];
        uint64_t n = nl->fi_off[i + 1] - nl->fi_off[i];
        for (uint64_t k = 0; k < n; k++) in[k] = g + nl->fi_idx[nl->fi_off[i] + k] * R;
        eval_vec(nl->type[i], in, n, gi, nr);
      }
    }
    for (uint64_t fi = j->f0; fi < j->f1; fi++) {
      const or_fault* f = &j->faults[fi];
      const uint64_t sv = f->value ? ~0ull : 0ull;
      for (uint64_t r = 0; r < nr; r++) {
        diff[r] = 0;
        svv[r] = sv;
      }
      epoch++;
      pend[f->site >> 6] |= 1ull << (f->site & 63);
      uint64_t npend = 1;
      for (uint64_t w = f->site >> 6; w < NW && npend; w++) {
        while (pend[w]) {
          const uint64_t i = w * 64 + (uint64_t)__builtin_ctzll(pend[w]);
          pend[w] &= pend[w] - 1;
          npend--;
          const uint64_t* gi = g + i * R;
          if (i == f->site && f->pin == 0) {
            for (uint64_t r = 0; r < nr; r++) v[r] = sv;
          } else {
            const uint64_t* in[4];
            uint64_t n = nl->fi_off[i + 1] - nl->fi_off[i];
            for (uint64_t k = 0; k < n; k++) {
              uint64_t d = nl->fi_idx[nl->fi_off[i] + k];
              in[k] = ((stamp[d] == epoch) ? b : g) + d * R;
            }
            if (i == f->site) in[f->pin - 1] = svv;
            eval_vec(nl->type[i], in, n, v, nr);
          }
          uint64_t changed = 0;
          for (uint64_t r = 0; r < nr; r++) changed |= v[r] ^ gi[r];
          if (!changed) continue; /* no difference leaves this element */
          memcpy(b + i * R, v, nr * 8);
          stamp[i] = epoch;
          if (i >= nl->po_begin)
            for (uint64_t r = 0; r < nr; r++) diff[r] |= (gi[r] ^ v[r]) & mask[r];
          for (uint64_t k = nl->fo_off[i]; k < nl->fo_off[i + 1]; k++) {
            const uint64_t c = nl->fo_idx[k];
            const uint64_t m = 1ull << (c & 63);
            if (!(pend[c >> 6] & m)) {
              pend[c >> 6] |= m;
              npend++;
            }
          }
        }
      }
      for (uint64_t r = 0; r < nr; r++)
        accumulate(&j->res[fi - j->base], diff[r], bitsv[r], c0 + r, W - 1);
    }
  }
  free(g);
  free(b);
  free(stamp);
  free(pend);
  free(v);
  free(diff);
  free(mask);
  free(bitsv);
  free(svv);
}

static void* job_main(void* arg) {
  job_t* j = arg;
  if (j->mode == 0)
    run_naive(j);
  else if (j->mode == 2)
    run_event_chunked(j);
  else
    run_event(j);
  return NULL;
}

void or_simulate(const or_netlist* nl, const or_fault* faults, uint64_t f0, uint64_t f1,
                 const uint64_t* words, uint64_t P, uint64_t rd0, uint64_t rd1, int mode,
                 int n_threads, or_result* res) {
  if (f1 <= f0) return;
  if (n_threads < 1) n_threads = 1;
  if ((uint64_t)n_threads > f1 - f0) n_threads = (int)(f1 - f0);
  job_t* jobs = calloc((size_t)n_threads, sizeof(job_t));
  pthread_t* th = calloc((size_t)n_threads, sizeof(pthread_t));
  uint64_t per = (f1 - f0 + (uint64_t)n_threads - 1) / (uint64_t)n_threads;
  for (int t = 0; t < n_threads; t++) {
    uint64_t a = f0 + (uint64_t)t * per, b = a + per;
    if (b > f1) b = f1;
    if (a > f1) a = f1;
    jobs[t] = (job_t){nl, faults, a, b, words, P, rd0, rd1, mode, res, f0};
    if (n_threads == 1)
      job_main(&jobs[t]);
    else
      pthread_create(&th[t], NULL, job_main, &jobs[t]);
  }
  if (n_threads > 1)
    for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  free(jobs);
  free(th);
}
