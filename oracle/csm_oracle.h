/* CPU restatement of ParaCOSM's continuous-subgraph-matching semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only
 * as the checker or the timed CPU baseline; the product path never calls it.
 *
 * Semantics restated (reference file:line, paths inside ParaCOSM/CSM):
 *   - per-update sequential loop ........ matching/main.cpp:628-674 (SingleThreadUpdate)
 *   - data graph mutation ............... graph/graph.cpp:58-116 (AddEdge / RemoveEdge)
 *   - GraphFlow matching orders ......... matching/GraphFlow/graphflow.cpp:36-169
 *   - edge-anchored backtracking ........ matching/GraphFlow/graphflow.cpp:181-265
 *   - insertion: count after adding ..... matching/GraphFlow/graphflow.cpp:289-355
 *   - deletion: count before removing ... matching/GraphFlow/graphflow.cpp:357-416
 *   - per-update result cap ............. matching/SymBi/symbi.cpp:583 (stop at exactly the cap)
 *   - label-triple safe test ............ matching/Parallel_GraphFlow/parallel_graphflow.cpp:1990-2016
 *   - DAG root / SymBi DAG .............. matching/SymBi/symbi.cpp:113-238
 *   - TurboFlux spanning tree ........... matching/TurboFlux/turboflux.cpp:69-219
 *   - d1 / d2 candidate flags ........... matching/SymBi/symbi.cpp:259-349, 404-469
 *   - CaLiG lighting after static filter  matching/Parallel_CaLiG/parallel_calig.cpp:337-429, 970-975
 *
 * Counts are the number of injective (unless homomorphism), label-preserving
 * embeddings of the query that contain the updated edge.  The match-set hash
 * is sum over embeddings of mix64(sum_q pair_hash(q, m[q])) mod 2^64, which
 * does not depend on enumeration order.  `bytes` is the canonical
 * algorithmic-byte figure: 4 B x sum over expanded search-tree nodes of the
 * sizes of all backward neighbour segments S(m[u_j], L(u), l(u,u_j)), in the
 * GraphFlow order of the anchor query edge, plus 16 B per applied edge
 * mutation.
 *
 * With want_hash = 0 the search is the engine's counting search: the
 * independent tail of each order (the longest suffix with no query edge
 * inside and no vertex label more than three times) is counted instead of
 * being enumerated: a product over label groups of injective assignments.  Counts are the
 * same; `bytes` then covers the nodes that search expands (each tail
 * position once per prefix, while the product is nonzero).
 */
#ifndef CSM_ORACLE_H
#define CSM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORACLE_OK = 0,
  ORACLE_CAPPED = 1,
  ORACLE_INVALID = 3
};

typedef struct oracle_update {  /* same 16-byte layout as csm_update */
  uint8_t type;   /* 'v' or 'e' */
  uint8_t is_add;
  uint16_t pad;
  uint32_t id1, id2, label;
} oracle_update;

typedef struct oracle_result {
  uint64_t pos, neg, hash, bytes;
  uint32_t status, safe;  /* safe = 1 when the label-triple test says no query edge can match */
} oracle_result;

/* Runs the whole stream in order.  Returns 0, or a negative value on bad input.
 * max_results = 0 means no cap.  homo != 0 drops the injectivity check. */
int oracle_run(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
               uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
               uint64_t n_up, const oracle_update* ups, uint64_t max_results, int homo,
               int want_hash, oracle_result* out);

/* Exhaustive brute-force count (every injective label-preserving map) of the
 * embeddings containing edge (v1, v2) in the given graph; for tiny inputs. */
int oracle_brute_count(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                       uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
                       uint32_t v1, uint32_t v2, int homo, uint64_t* count, uint64_t* hash);

/* GraphFlow matching orders of the query (graphflow.cpp:36-169): order[i*n_qv + j]
 * is the j-th query vertex of the order anchored on the i-th query edge. */
int oracle_graphflow_orders(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                            uint32_t* order);

/* Candidate index (the d1 / d2 flags) of the TurboFlux plugin (a DCG over a
 * query spanning tree, ParaCOSM/CSM/matching/TurboFlux/turboflux.cpp:69-331)
 * or the SymBi plugin (a DCS over a DAG of every query edge,
 * SymBi/symbi.cpp:113-349).  The DAG is chosen on the graph before the
 * stream; the flags are those of the graph after the first n_up updates.
 * Outputs: root, order[n_qv] (serialized tree), parents[n_qv] (bitmask of DAG
 * parents), d1 / d2 as [n_qv][words] bitsets over data vertex ids.  Returns
 * the number of data vertex ids, or a negative value on bad input. */
enum { ORACLE_INDEX_TURBOFLUX = 1, ORACLE_INDEX_SYMBI = 2 };

/* Number of embeddings of the query in the graph after the first n_up
 * updates (InitialMatching, ParaCOSM/CSM/matching/GraphFlow/graphflow.cpp:268-284). */
int oracle_initial_count(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                         uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
                         uint64_t n_up, const oracle_update* ups, int homo, uint64_t* count);
int oracle_index(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                 uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
                 uint64_t n_up, const oracle_update* ups, int algo, uint32_t* root, uint32_t* order,
                 uint32_t* parents, uint64_t words, uint64_t* d1, uint64_t* d2);

/* Injective assignments of a group of g <= 3 same-label tail positions (the
 * counting search's group count), from N[M] = the number of candidates whose
 * membership set over the group is exactly M (N[0] unused); without
 * injectivity under homo.  Saturates at 2^58. */
uint64_t oracle_group_assignments(uint32_t g, const uint64_t* N, int homo);

/* CaLiG-style candidate flags on the graph after the first n_up updates, as
 * [n_qv][words] bitsets (any output may be null):
 *   li0: L(v) = L(u) and v has, per (vertex label, edge label) pair of u's
 *        query edges, at least as many neighbours as u (one under homo);
 *   li1: li0 and every query neighbour of u has an li0 neighbour of v;
 *   lit: the lighting of the reference's CaLiG after static filtering
 *        (ParaCOSM/CSM/matching/Parallel_CaLiG/parallel_calig.cpp:337-429,
 *        970-975): the greatest set where every lit (u, v) maps u's query
 *        neighbours to distinct lit neighbours of v.
 * lit is contained in li1.  Returns the number of data vertex ids. */
int oracle_calig_index(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                       uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
                       uint64_t n_up, const oracle_update* ups, int homo, uint64_t words, uint64_t* li0,
                       uint64_t* li1, uint64_t* lit);

#ifdef __cplusplus
}
#endif
#endif
