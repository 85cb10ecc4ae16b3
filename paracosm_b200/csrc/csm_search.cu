// Search kernels: seeding, the warp-cooperative expansion, finalisation.
//
// Reference semantics restated (paths inside ParaCOSM/CSM):
//   seeds of an edge update ......... matching/GraphFlow/graphflow.cpp:305-352 (each query
//                                     edge whose label triple matches, both orientations)
//   candidate generation / join ..... matching/GraphFlow/graphflow.cpp:181-265 (label filter,
//                                     adjacency to every matched query neighbour, injectivity)
//   index filter (TurboFlux/SymBi) .. matching/SymBi/symbi.cpp:516 (candidate must have d2 set)
//   per-update cap .................. matching/SymBi/symbi.cpp:583 (stop at exactly the cap)
//   Classify (safe update) .......... matching/Parallel_GraphFlow/parallel_graphflow.cpp:1990-2016
//
// Expansion scheme.  A warp owns one root task (update, anchor edge,
// orientation) at a time and walks its search tree depth first, but each
// level holds up to 32 partial matches at once: to extend level d the warp
// takes the next 32 (entry, driver element) pairs of level d's entries -- the
// driver being the smallest back-neighbour segment -- so lanes stay busy even
// when segments are a few elements long.  Every lane checks its candidate
// against the other back-neighbour segments (binary search), the same-label
// matched vertices (injectivity), the candidate filter, and the batch-time
// presence of every back edge; survivors are compacted with a ballot into
// level d + 1 together with the driver segment of their own next level
// (an empty next-level segment prunes them right away).  Leaves are only
// counted.
#include "csm_kernels.cuh"

namespace csm {

struct LevelSM {
  uint32_t v[32];     // data vertex of this level's position
  uint32_t dlo[32];   // driver segment of the next position: pool offset
  uint32_t dn[32];    //   and length
  uint8_t par[32];    // entry index in the previous level
  uint8_t dsel[32];   // back entry that is the driver
  uint32_t cnt, cur_e, cur_k, pad;
};

size_t search_smem_bytes(uint32_t n_q, uint32_t warps) {
  const uint32_t levels = n_q > 2 ? n_q - 2 : 1;
  return (size_t)warps * levels * sizeof(LevelSM);
}

__device__ __forceinline__ bool d2_bit(const uint64_t* d2, uint64_t words, uint32_t q, uint32_t v) {
  return (d2[(uint64_t)q * words + (v >> 6)] >> (v & 63)) & 1ULL;
}

__global__ void k_seed(uint32_t B, const UpdInfo* info, DevGraph g, const Plan* plan, const uint64_t* d2,
                       uint64_t d2_words, Task* tasks, unsigned int* n_tasks, uint32_t task_cap,
                       uint32_t* safe, unsigned int* error) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  const UpdInfo u = info[s];
  uint32_t sf = 1;
  if ((u.flags & UF_VALID) && !(u.flags & UF_INVALID)) {
    const uint32_t L1 = g.vlabel[u.v1], L2 = g.vlabel[u.v2], l = u.label;
    const uint32_t na = plan->n_anchor;
    for (uint32_t a = 0; a < na; a++) {
      const PlanAnchor* A = &plan->anchors[a];
      if (A->el != l) continue;
      const bool o0 = A->la == L1 && A->lb == L2;
      const bool o1 = A->la == L2 && A->lb == L1;
      if (!(o0 || o1)) continue;
      sf = 0;
      for (int o = 0; o < 2; o++) {
        if (!(o ? o1 : o0)) continue;
        const uint32_t x = o ? u.v2 : u.v1, y = o ? u.v1 : u.v2;
        if (d2 && !(d2_bit(d2, d2_words, A->pos[0].qv, x) && d2_bit(d2, d2_words, A->pos[1].qv, y))) continue;
        unsigned int i = atomicAdd(n_tasks, 1u);
        if (i >= task_cap) { atomicExch(error, kErrTaskOverflow); continue; }
        tasks[i] = Task{s, (uint16_t)a, (uint8_t)o, 0};
      }
    }
  }
  safe[s] = sf;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= (uint32_t)o) v += t;
  }
  return v;
}

// Full candidate check of data vertex x for position `pos` given the matched
// prefix m[0 .. pos-1]; `dsel` is the back entry whose segment produced x.
__device__ __forceinline__ bool check_candidate(const SearchParams& p, const uint32_t* pool, const PlanAnchor* A,
                                                uint32_t pos, uint32_t x, const uint32_t* m, uint32_t dsel,
                                                int32_t t) {
  const PlanPos P = A->pos[pos];
  if (!p.homo) {
    for (uint32_t mk = P.samelab; mk; mk &= mk - 1) {
      if (m[__ffs(mk) - 1] == x) return false;
    }
  }
  if (p.d2 && !d2_bit(p.d2, p.d2_words, P.qv, x)) return false;
  for (uint32_t b = 0; b < P.nb; b++) {
    const uint32_t j = A->back_pos[P.boff + b], c = A->back_combo[P.boff + b];
    const uint32_t v = m[j];
    if (b != dsel) {
      uint64_t lo, hi;
      segment(p.g, v, c, lo, hi);
      if (!contains_u32(pool, lo, hi, x)) return false;
    }
    if (!present_at(p.g, v, c, x, t)) return false;
  }
  return true;
}

// Driver segment of position np for prefix m (the smallest union-graph back
// segment); false if some back segment is empty at batch time t.  `bytes`
// receives 4 B x the sizes at time t of all back segments: the algorithmic
// bytes of expanding this node.
__device__ __forceinline__ bool pick_driver(const SearchParams& p, const PlanAnchor* A, uint32_t np,
                                            const uint32_t* m, int32_t t, uint32_t& dlo, uint32_t& dn,
                                            uint32_t& dsel, unsigned long long& bytes) {
  const PlanPos P = A->pos[np];
  uint32_t best = 0xffffffffu;
  bool empty = false;
  unsigned long long b4 = 0;
  for (uint32_t b = 0; b < P.nb; b++) {
    const uint32_t j = A->back_pos[P.boff + b], c = A->back_combo[P.boff + b];
    uint64_t lo, hi;
    segment(p.g, m[j], c, lo, hi);
    const uint32_t sz = (uint32_t)(hi - lo);
    const uint32_t szt = seg_size_at(p.g, m[j], c, lo, hi, t);
    b4 += 4ull * szt;
    if (szt == 0) empty = true;
    if (sz < best) { best = sz; dsel = b; dlo = (uint32_t)lo; }
  }
  dn = best;
  bytes = b4;
  return !empty;
}

template <int W>
__global__ void __launch_bounds__(W * 32) k_search(SearchParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t n = p.plan->n;
  const uint32_t nlev = n > 2 ? n - 2 : 1;
  LevelSM* lv = reinterpret_cast<LevelSM*>(smem_raw) + (size_t)warp * nlev - 1;  // levels 1 .. n-2
  const uint32_t* pool = p.g.pools[p.g.ps->active];
  const uint32_t ntask = min(*p.n_tasks, p.task_cap);
  volatile unsigned int* stop = p.stop;

  for (;;) {
    uint32_t ti = 0;
    if (lane == 0) ti = atomicAdd(p.task_next, 1u);
    ti = __shfl_sync(0xffffffffu, ti, 0);
    if (ti >= ntask) break;
    const Task T = p.tasks[ti];
    const uint32_t t = T.upd;
    if (stop[t]) continue;
    const PlanAnchor* A = &p.plan->anchors[T.anchor];
    const UpdInfo U = p.info[t];
    const uint32_t m0 = T.orient ? U.v2 : U.v1, m1 = T.orient ? U.v1 : U.v2;
    unsigned long long cnt_local = 0, hash_local = 0, bytes_local = 0;

    if (n == 2) {
      if (lane == 0) {
        cnt_local = 1;
        if (p.want_hash) hash_local = mix64(pair_hash(A->pos[0].qv, m0) + pair_hash(A->pos[1].qv, m1));
      }
    } else {
      // driver of position 2 for the root (positions 0 and 1 matched)
      const PlanPos P2 = A->pos[2];
      uint32_t sz = 0xffffffffu, szt = 1;
      uint64_t lo = 0, hi = 0;
      unsigned long long rb = 0;
      if (lane < P2.nb) {
        const uint32_t j = A->back_pos[P2.boff + lane], c = A->back_combo[P2.boff + lane];
        const uint32_t v = j == 0 ? m0 : m1;
        segment(p.g, v, c, lo, hi);
        sz = (uint32_t)(hi - lo);
        szt = seg_size_at(p.g, v, c, lo, hi, (int32_t)t);
        rb = 4ull * szt;
      }
      const bool root_empty = __any_sync(0xffffffffu, szt == 0);
#pragma unroll
      for (int o = 16; o; o >>= 1) rb += __shfl_xor_sync(0xffffffffu, rb, o);
      bytes_local += rb;
      uint64_t key = ((uint64_t)sz << 32) | lane;
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        uint64_t other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other < key ? other : key;
      }
      const uint32_t minsz = root_empty ? 0u : (uint32_t)(key >> 32), sel = (uint32_t)key;
      const uint32_t dlo0 = (uint32_t)__shfl_sync(0xffffffffu, lo, sel);
      if (minsz != 0) {
        if (lane == 0) {
          lv[1].cnt = 1; lv[1].cur_e = 0; lv[1].cur_k = 0;
          lv[1].dlo[0] = dlo0; lv[1].dn[0] = minsz; lv[1].dsel[0] = (uint8_t)sel;
        }
        __syncwarp();
        int d = 1;
        uint32_t iter = 0;
        while (d >= 1) {
          if ((++iter & 7) == 0) {
            uint32_t st = (lane == 0) ? stop[t] : 0u;
            if (__shfl_sync(0xffffffffu, st, 0)) break;
          }
          LevelSM& L = lv[d];
          const uint32_t cnt = L.cnt, ce = L.cur_e, ck = L.cur_k;
          if (ce >= cnt) { d--; continue; }
          // the next 32 (entry, driver element) pairs of this level
          const uint32_t el = ce + lane;
          const uint32_t rem = (el < cnt) ? L.dn[el] - (lane == 0 ? ck : 0u) : 0u;
          const uint32_t incl = warp_incl_scan(rem, lane);
          const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
          uint32_t owner = 0;
#pragma unroll
          for (uint32_t step = 16; step; step >>= 1) {
            const uint32_t v = __shfl_sync(0xffffffffu, incl, owner + step - 1);
            if (v <= lane) owner += step;
          }
          const uint32_t prev = __shfl_sync(0xffffffffu, incl, owner > 0 ? (owner - 1) & 31 : 0);
          const bool active = lane < total;
          const uint32_t e = ce + owner;
          const uint32_t kk = lane - (owner > 0 ? prev : 0u) + (owner == 0 ? ck : 0u);
          uint32_t nce, nck;
          if (total <= 32) {
            nce = ce + min(32u, cnt - ce); nck = 0;
          } else {
            const uint32_t o31 = __shfl_sync(0xffffffffu, owner, 31);
            const uint32_t k31 = __shfl_sync(0xffffffffu, kk, 31);
            const uint32_t e31 = ce + o31;
            if (k31 + 1 >= L.dn[e31]) { nce = e31 + 1; nck = 0; } else { nce = e31; nck = k31 + 1; }
          }
          const uint32_t pos = (uint32_t)d + 1;
          bool valid = false;
          uint32_t x = 0, ndlo = 0, ndn = 0, ndsel = 0;
          unsigned long long nb4 = 0;
          uint32_t m[kMaxQ];
          if (active) {
            x = pool[(uint64_t)L.dlo[e] + kk];
            m[0] = m0; m[1] = m1;
            uint32_t idx = e;
            for (int l2 = d; l2 >= 2; --l2) { m[l2] = lv[l2].v[idx]; idx = lv[l2].par[idx]; }
            valid = check_candidate(p, pool, A, pos, x, m, L.dsel[e], (int32_t)t);
            if (valid && pos + 1 < n) {
              m[pos] = x;
              valid = pick_driver(p, A, pos + 1, m, (int32_t)t, ndlo, ndn, ndsel, nb4);
            }
          }
          __syncwarp();
          if (lane == 0) { L.cur_e = nce; L.cur_k = nck; }
          const uint32_t mask = __ballot_sync(0xffffffffu, valid);
          if (pos + 1 < n) {
#pragma unroll
            for (int o = 16; o; o >>= 1) nb4 += __shfl_xor_sync(0xffffffffu, nb4, o);
            bytes_local += nb4;
          }
          if (pos == n - 1) {
            const uint32_t c = __popc(mask);
            if (p.want_hash) {
              unsigned long long h = 0;
              if (valid) {
                uint64_t s = pair_hash(A->pos[pos].qv, x);
                for (uint32_t q = 0; q < pos; q++) s += pair_hash(A->pos[q].qv, m[q]);
                h = mix64(s);
              }
#pragma unroll
              for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
              hash_local += h;
            }
            cnt_local += c;
            if (c && p.cap) {
              unsigned int hit = 0;
              if (lane == 0) {
                const unsigned long long old = atomicAdd(&p.count[t], cnt_local);
                cnt_local = 0;
                if (old + c >= p.cap) { stop[t] = 1u; hit = 1; }
              }
              if (__shfl_sync(0xffffffffu, hit, 0)) break;
            }
          } else {
            LevelSM& N = lv[pos];
            if (valid) {
              const uint32_t slot = __popc(mask & ((1u << lane) - 1u));
              N.v[slot] = x; N.par[slot] = (uint8_t)e; N.dlo[slot] = ndlo; N.dn[slot] = ndn;
              N.dsel[slot] = (uint8_t)ndsel;
            }
            if (lane == 0) { N.cnt = __popc(mask); N.cur_e = 0; N.cur_k = 0; }
            __syncwarp();
            if (mask) d = (int)pos;
          }
        }
      }
    }
    if (lane == 0) {
      if (cnt_local) {
        const unsigned long long old = atomicAdd(&p.count[t], cnt_local);
        if (p.cap && old + cnt_local >= p.cap) stop[t] = 1u;
      }
      if (p.want_hash && hash_local) atomicAdd(&p.hash[t], hash_local);
      if (bytes_local) atomicAdd(&p.bytes[t], bytes_local);
    }
    __syncwarp();
  }
}

void launch_search(const SearchParams& p, uint32_t n_q, uint32_t blocks, uint32_t warps, cudaStream_t s) {
  const size_t smem = search_smem_bytes(n_q, warps);
  switch (warps) {
    case 4:
      cudaFuncSetAttribute(k_search<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_search<4><<<blocks, 4 * 32, smem, s>>>(p);
      break;
    case 16:
      cudaFuncSetAttribute(k_search<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_search<16><<<blocks, 16 * 32, smem, s>>>(p);
      break;
    default:
      cudaFuncSetAttribute(k_search<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_search<8><<<blocks, 8 * 32, smem, s>>>(p);
      break;
  }
}

__global__ void k_finalize(uint32_t B, const UpdInfo* info, const unsigned long long* count,
                           const unsigned long long* hash, const unsigned long long* bytes, const uint32_t* safe,
                           uint64_t cap, int want_hash, csm_result* out) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  const UpdInfo u = info[s];
  csm_result r;
  r.pos = 0; r.neg = 0; r.hash = 0; r.work_bytes = 0; r.latency_ns = 0;
  r.status = CSM_ST_OK; r.safe = safe ? safe[s] : 1u;
  if ((u.flags & UF_INVALID) || !(u.flags & UF_VALID)) {
    r.status = (u.flags & UF_INVALID) ? CSM_ST_INVALID : CSM_ST_OK;  // vertex updates count nothing
    r.safe = 1;
  } else {
    unsigned long long c = count[s];
    if (cap && c >= cap) { c = cap; r.status = CSM_ST_CAPPED; }
    if (u.flags & UF_ADD) r.pos = c; else r.neg = c;
    if (want_hash && r.status == CSM_ST_OK) r.hash = hash[s];
    r.work_bytes = (bytes ? bytes[s] : 0ull) + ((u.flags & UF_MUT) ? 16ull : 0ull);
  }
  out[s] = r;
}

__global__ void k_classify(uint64_t n, const csm_update* ups, DevGraph g, const Plan* plan, uint8_t* safe) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const csm_update u = ups[i];
  uint8_t sf = 1;
  if (u.id1 < g.n && u.id2 < g.n) {
    const uint32_t L1 = g.vlabel[u.id1], L2 = g.vlabel[u.id2];
    for (uint32_t a = 0; a < plan->n_anchor && sf; a++) {
      const PlanAnchor* A = &plan->anchors[a];
      if (A->el == u.label && ((A->la == L1 && A->lb == L2) || (A->la == L2 && A->lb == L1))) sf = 0;
    }
  }
  safe[i] = sf;
}

}  // namespace csm
