/*
 * p2c_b200.h — C ABI of the B200 (sm_100a) certification hot path of P2C-CCD.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns an
 * int status (P2C_OK = 0) and leaves a message for p2c_last_error() on failure.
 * Pointers named `*_dev` are device pointers; `*_host` are host pointers.  All
 * device work is issued on the caller's `stream` (a cudaStream_t passed as
 * void*, NULL = legacy default stream) and is asynchronous unless the entry
 * point says otherwise.
 *
 * Record layouts are byte-identical to the reference's host structs so that a
 * std::vector of reference primitives can be handed over without repacking:
 *   p2c_point_triangle == p2cccd::PointTriangleIntervalPrimitive (240 B)
 *   p2c_edge_edge      == p2cccd::EdgeEdgeIntervalPrimitive      (240 B)
 *   p2c_interval_result== p2cccd::PrimitiveIntervalResult        (72 B)
 * (reference: src/cpp/certificate/certificate_engine.h:32-81).
 */
#ifndef P2C_B200_H_
#define P2C_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define P2C_OK 0
#define P2C_ERR_INVALID 1  /* invalid argument; the reference raises ValueError */
#define P2C_ERR_CUDA 2     /* a CUDA runtime call failed */
#define P2C_ERR_CAPACITY 3 /* an output buffer was too small; required size reported */
#define P2C_ERR_TIMEOUT 4  /* a bounded device wait gave up (error word set) */

/* CertificateStatus (reference: src/cpp/common/runtime_contracts.h:20-24) */
#define P2C_STATUS_COLLISION 0
#define P2C_STATUS_SEPARATION 1
#define P2C_STATUS_UNDECIDED 2

/* ExactFeatureFamilyMask (reference: certificate_engine.h:12-15) */
#define P2C_FAMILY_POINT_TRIANGLE 1u
#define P2C_FAMILY_EDGE_EDGE 2u

/* CertificateReasonCode (reference: certificate_engine.h:17-22) */
#define P2C_REASON_NONE 0
#define P2C_REASON_MISSING_GEOMETRY 1
#define P2C_REASON_MAX_SUBDIVISION_DEPTH 2
#define P2C_REASON_INVALID_INPUT 3

/* CertificateRefinementMode (reference: runtime_contracts.h:26-31) */
#define P2C_REFINE_NONE 0
#define P2C_REFINE_BISECT_INTERVAL 1
#define P2C_REFINE_REQUEST_GEOMETRY 2
#define P2C_REFINE_ESCALATE_PRECISION 3

/* ---- records ------------------------------------------------------------ */
typedef struct p2c_trajectory {            /* LinearVertexTrajectory, 56 B */
  int64_t feature_id;
  double position_t0[3];
  double position_t1[3];
} p2c_trajectory;

typedef struct p2c_point_triangle {        /* PointTriangleIntervalPrimitive, 240 B */
  int64_t point_id;
  int64_t triangle_id;
  p2c_trajectory point;
  p2c_trajectory triangle_v0;
  p2c_trajectory triangle_v1;
  p2c_trajectory triangle_v2;
} p2c_point_triangle;

typedef struct p2c_edge_edge {             /* EdgeEdgeIntervalPrimitive, 240 B */
  int64_t edge_a_id;
  int64_t edge_b_id;
  p2c_trajectory edge_a0;
  p2c_trajectory edge_a1;
  p2c_trajectory edge_b0;
  p2c_trajectory edge_b1;
} p2c_edge_edge;

typedef struct p2c_interval_result {       /* PrimitiveIntervalResult, 72 B */
  uint8_t status;                          /* P2C_STATUS_* */
  uint8_t pad0[3];
  uint32_t covered_feature_mask;
  double interval_t0;
  double interval_t1;
  double toi_upper;
  double safe_margin_lb;
  uint8_t witness_family;
  uint8_t pad1[7];
  int64_t witness_id_a;
  int64_t witness_id_b;
  uint16_t reason_code;
  uint8_t next_refinement_mode;
  uint8_t pad2[5];
} p2c_interval_result;

typedef struct p2c_cert_config {           /* CertificateEngineConfig */
  double eps_time;
  double eps_space;
  uint16_t max_subdivision_depth;
  uint16_t pad[3];
} p2c_cert_config;

/* Aggregated work-item certificate, the reduction CertificateEngine::Evaluate
 * performs over its VF then EE primitive lists (certificate_engine.cpp:729-824). */
typedef struct p2c_query_certificate {
  uint8_t status;
  uint8_t witness_family;
  uint16_t reason_code;
  uint32_t covered_feature_mask;
  double toi_upper;
  double safe_margin_lb;
  int64_t witness_id_a;
  int64_t witness_id_b;
  int64_t witness_index;                   /* position of the witness primitive in its list, -1 if none */
  uint8_t next_refinement_mode;
  uint8_t pad[7];
} p2c_query_certificate;

/* Device-side counters of one certification launch. */
typedef struct p2c_certify_stats {
  uint64_t nodes_evaluated;                /* interval nodes whose mid sample was evaluated */
  uint64_t distance_evals;                 /* distance evaluations (3 per root + 1 per child) */
  uint64_t fp64_ops;                       /* counted FP64 add/sub/mul/div/sqrt (census launches only) */
  uint64_t donations;                      /* subtrees handed between lanes of a warp */
  uint64_t queries;                        /* queries certified */
  uint64_t error_word;                     /* nonzero if a bounded wait or a capacity check failed */
  uint64_t max_warp_iterations;            /* longest warp loop (one distance sample per lane per iteration) */
  uint64_t busy_lane_iterations;           /* sum over iterations of lanes holding work */
} p2c_certify_stats;

/* ---- library ------------------------------------------------------------ */
const char* p2c_last_error(void);
int p2c_abi_version(void);
/* Replaces IsCudaExactBuilt (src/cpp/certificate/certificate_cuda.h:10). */
int p2c_is_cuda_exact_built(void);
/* Device properties the kernels are sized from (SM count, smem per block). */
int p2c_device_info(int* sm_count, int* max_smem_per_block, int* cc_major, int* cc_minor);

/* ---- narrow phase: batch interval certificates ------------------------- */
/* Scratch bytes the device entry points below need for a batch of n primitives. */
size_t p2c_certify_workspace_bytes(int64_t n);

/* Replaces EvaluatePointTriangleBatchCuda (certificate_cuda.h:11-15), with
 * device pointers, a caller stream and caller-owned scratch.  Results are
 * bit-identical to EvaluatePointTriangleInterval (certificate_engine.cpp:481-515)
 * applied to each primitive.  stats_dev may be NULL. */
int p2c_certify_pt_batch(const p2c_point_triangle* prims_dev, int64_t n,
                         double interval_t0, double interval_t1,
                         const p2c_cert_config* config,
                         p2c_interval_result* results_dev,
                         void* workspace_dev, size_t workspace_bytes,
                         p2c_certify_stats* stats_dev, void* stream);

/* Replaces EvaluateEdgeEdgeBatchCuda (certificate_cuda.h:16-20). */
int p2c_certify_ee_batch(const p2c_edge_edge* prims_dev, int64_t n,
                         double interval_t0, double interval_t1,
                         const p2c_cert_config* config,
                         p2c_interval_result* results_dev,
                         void* workspace_dev, size_t workspace_bytes,
                         p2c_certify_stats* stats_dev, void* stream);

/* Both families in one persistent launch (point-triangle list, then
 * edge-edge list, as CrossCheckCpuCudaExact takes them, certificate_cuda.h:21-26);
 * each result equals the single-family entry points'.  Either list may be empty. */
int p2c_certify_batch2(const p2c_point_triangle* pt_dev, int64_t n_pt,
                       const p2c_edge_edge* ee_dev, int64_t n_ee,
                       double interval_t0, double interval_t1,
                       const p2c_cert_config* config,
                       p2c_interval_result* pt_results_dev,
                       p2c_interval_result* ee_results_dev,
                       void* workspace_dev, size_t workspace_bytes,
                       p2c_certify_stats* stats_dev, void* stream);

/* Host-buffer forms with the reference's ownership model (host-owned arrays,
 * synchronous, library-managed device memory): the drop-in for the pybind
 * `evaluate_point_triangle_batch_cuda` / `evaluate_edge_edge_batch_cuda`
 * (src/cpp/bindings/py_module.cpp:1972-1983).  n == 0 returns P2C_OK. */
int p2c_certify_pt_batch_host(const p2c_point_triangle* prims_host, int64_t n,
                              double interval_t0, double interval_t1,
                              const p2c_cert_config* config,
                              p2c_interval_result* results_host);
int p2c_certify_ee_batch_host(const p2c_edge_edge* prims_host, int64_t n,
                              double interval_t0, double interval_t1,
                              const p2c_cert_config* config,
                              p2c_interval_result* results_host);

/* The library's CPU certifier, the CPU side of CrossCheckCpuCudaExact
 * (certificate_cuda.cu:616-679): EvaluatePointTriangleInterval /
 * EvaluateEdgeEdgeInterval (certificate_engine.cpp:300-386, 481-551) on the
 * host's cores, host arrays in and out.  Same validation messages as the GPU
 * entry points.  It shares only the distance and motion formulas with the
 * device; the GPU entry points never call it. */
int p2c_certify_pt_batch_cpu(const p2c_point_triangle* prims_host, int64_t n,
                             double interval_t0, double interval_t1,
                             const p2c_cert_config* config,
                             p2c_interval_result* results_host);
int p2c_certify_ee_batch_cpu(const p2c_edge_edge* prims_host, int64_t n,
                             double interval_t0, double interval_t1,
                             const p2c_cert_config* config,
                             p2c_interval_result* results_host);

/* Census launch: the same certifier with lane-local depth-first order (the
 * reference's node set exactly) and FP64 operation counting.  Used to state the
 * algorithmic FP64 work of a batch; not a production path. */
int p2c_certify_census(const p2c_point_triangle* pt_dev, int64_t n_pt,
                       const p2c_edge_edge* ee_dev, int64_t n_ee,
                       double interval_t0, double interval_t1,
                       const p2c_cert_config* config,
                       p2c_interval_result* pt_results_dev,
                       p2c_interval_result* ee_results_dev,
                       void* workspace_dev, size_t workspace_bytes,
                       p2c_certify_stats* stats_dev, void* stream);

/* ---- work queues: many work items in one launch --------------------------- */
size_t p2c_certify_queries_workspace_bytes(int64_t n_queries);

/* CertificateEngine::Evaluate (certificate_engine.cpp:729-824) for every work
 * item of a queue (ProcessExactWorkQueueCpu, :593-661) in one launch.  The
 * queue's primitives are two flat record lists; pt_query/ee_query give each
 * primitive's work-item index (non-decreasing; a work item's primitives are
 * contiguous and in its list order) and pt_offsets/ee_offsets (n_queries + 1)
 * the same as CSR offsets.  Each work item has its interval (q_t0, q_t1,
 * already validated) and feature_family_mask; only primitives of requested
 * families may be listed.  certs_dev[q] is the work item's certificate; a
 * primitive failing validation before the first collision makes it undecided
 * with reason InvalidInput, as the work queue reports an Evaluate error
 * (:629-632).  One CertificateEngineConfig for the whole call. */
int p2c_certify_queries(const p2c_point_triangle* pt_dev, int64_t n_pt, const int64_t* pt_query_dev,
                        const p2c_edge_edge* ee_dev, int64_t n_ee, const int64_t* ee_query_dev,
                        int64_t n_queries, const int64_t* pt_offsets_dev, const int64_t* ee_offsets_dev,
                        const double* q_t0_dev, const double* q_t1_dev, const uint32_t* q_mask_dev,
                        const p2c_cert_config* config,
                        p2c_interval_result* pt_results_dev, p2c_interval_result* ee_results_dev,
                        p2c_query_certificate* certs_dev,
                        void* workspace_dev, size_t workspace_bytes,
                        p2c_certify_stats* stats_dev, void* stream);

/* Work queues for callers that cannot allocate device memory — code running
 * while a CUDA graph is captured, frame loops that forbid allocation, hosts that
 * own all device memory under a fixed budget.  No counterpart in the reference.
 * Same arguments and results as p2c_certify_queries without the workspace: the
 * scratch is a 1 MiB file-scope device array that every GPU loading this library
 * holds until exit, so at most P2C_STATIC_QUEUE_MAX_QUERIES work items per call
 * (larger queues return P2C_ERR_INVALID).  The first call on a device resolves
 * the array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  Later calls made outside capture resolve it again (a
 * device reset can move the array).  Each call clears the scratch it uses before reading it,
 * but all calls on a device share the one array: calls that overlap on the GPU
 * (different streams, or host threads without ordering) race and must not be
 * issued.  It calls no cudaMalloc, cudaFree or allocating library routine. */
#define P2C_STATIC_QUEUE_MAX_QUERIES 26000
int p2c_certify_queries_static(const p2c_point_triangle* pt_dev, int64_t n_pt, const int64_t* pt_query_dev,
                               const p2c_edge_edge* ee_dev, int64_t n_ee, const int64_t* ee_query_dev,
                               int64_t n_queries, const int64_t* pt_offsets_dev, const int64_t* ee_offsets_dev,
                               const double* q_t0_dev, const double* q_t1_dev, const uint32_t* q_mask_dev,
                               const p2c_cert_config* config,
                               p2c_interval_result* pt_results_dev, p2c_interval_result* ee_results_dev,
                               p2c_query_certificate* certs_dev,
                               p2c_certify_stats* stats_dev, void* stream);

/* ---- scenes: swept-AABB candidates and their certificates ----------------- */
/* A scene: vertex trajectories over one step plus topology, all device arrays.
 * Objects are connected components (the scene tool's DSU objects,
 * scene_object_envelope_native_ti_walltime.cpp:497-520) or whole meshes. */
typedef struct p2c_scene {
  const double* v_t0;        /* nv x 3 positions at t = 0 */
  const double* v_t1;        /* nv x 3 positions at t = 1 */
  const int32_t* faces;      /* nf x 3 vertex indices */
  const int32_t* edges;      /* ne x 2 vertex indices (unique edges) */
  const int32_t* v_obj;      /* nv object ids; < 0 = vertex in no face (never a candidate) */
  const int32_t* f_obj;      /* nf object ids */
  const int32_t* e_obj;      /* ne object ids */
  int64_t nv, nf, ne;
  double thickness;          /* >= 0, added to every swept box (Expand, :263-270) */
  int32_t exclude_self;      /* 1: no candidate inside one object (mesh-pair queries) */
  int32_t n_obj;             /* object ids lie in [0, n_obj); with exclude_self and
                                1 <= n_obj <= 64, primitives outside every other object's
                                swept box are culled first (the scene tool's object
                                envelopes, :521-545); 0 = no culling */
} p2c_scene;

/* Workspace of p2c_scene_candidates for the given sizes and pair capacities. */
size_t p2c_scene_candidates_workspace_bytes(int64_t nv, int64_t nf, int64_t ne, int64_t vf_cap, int64_t ee_cap);

/* Swept-AABB candidate pairs of a scene by sweep-and-prune.  Replaces the
 * pair loops of BuildMeshExactCertificateQuery (cpp/certificate/
 * mesh_exact_query.cpp:211-317) and the scene tool's SweepPairs /
 * BuildVFCandidates / BuildEECandidates (tools/scene_object_envelope_native_
 * ti_walltime.cpp:603-699) with the same pair set.  Pairs are written as
 * (vertex << 32 | face) and (edge_lo << 32 | edge_hi); counts_dev[0..3] =
 * {vf pairs, ee pairs, error word (1: non-finite coordinate), sweep axis}.
 * When a count exceeds its capacity only capacity pairs are kept and the
 * caller retries with a larger buffer (counts are the full totals).
 * sort_pairs = 1 sorts each list ascending, padding with ~0 up to its
 * capacity: the order BuildMeshExactCertificateQuery emits its primitives. */
int p2c_scene_candidates(const p2c_scene* scene, uint64_t* vf_pairs_dev, int64_t vf_cap,
                         uint64_t* ee_pairs_dev, int64_t ee_cap, uint64_t* counts_dev,
                         int sort_pairs, void* workspace_dev, size_t workspace_bytes, void* stream);

/* Aggregate of a scene certification: the CertificateEngine::Evaluate
 * reduction (certificate_engine.cpp:729-824) over the VF list then the EE list
 * in pair order, plus per-status counts and the undecided (fallback-replay)
 * queue length. */
typedef struct p2c_scene_summary {
  p2c_query_certificate query;
  uint64_t collisions, separations, undecided;
  uint64_t vf_certified, ee_certified;
  uint64_t undecided_queued;                /* this scene's undecided entries (written or dropped) */
  uint64_t error_word;                      /* 1: time budget, 2: pair overflow, 4: invalid geometry,
                                               8: undecided queue full (entries of this scene dropped) */
} p2c_scene_summary;

size_t p2c_scene_certify_workspace_bytes(void);

/* Certificates of every candidate pair (the scene tool's every-candidate
 * rows, RunAllExactRows :1239-1281, with the reference certifier instead of
 * the external exact kernel).  n per family = min(counts_dev[k], cap) read on
 * the device, so this can follow p2c_scene_candidates without a host sync.
 * Results are positional with the pair lists.  Undecided candidates are
 * appended to undecided_queue_dev as (family << 63 | pair position) when it is
 * non-NULL (capacity undecided_cap); entries past the capacity are counted in
 * undecided_queued but not written, and set bit 8 of the summary's error word
 * (the caller re-runs with a larger queue).  summary_dev may be NULL. */
int p2c_scene_certify(const p2c_scene* scene, const uint64_t* vf_pairs_dev, int64_t vf_cap,
                      const uint64_t* ee_pairs_dev, int64_t ee_cap, const uint64_t* counts_dev,
                      double interval_t0, double interval_t1, const p2c_cert_config* config,
                      uint32_t family_mask,
                      p2c_interval_result* vf_results_dev, p2c_interval_result* ee_results_dev,
                      uint64_t* undecided_queue_dev, int64_t undecided_cap,
                      p2c_scene_summary* summary_dev,
                      void* workspace_dev, size_t workspace_bytes, void* stream);

/* Materialise candidate pairs as reference primitive records (the output
 * list of BuildMeshExactCertificateQuery): ids are scene indices, trajectory
 * feature ids are vertex indices. */
int p2c_scene_materialize(const p2c_scene* scene, const uint64_t* vf_pairs_dev, int64_t n_vf,
                          const uint64_t* ee_pairs_dev, int64_t n_ee,
                          p2c_point_triangle* vf_records_dev, p2c_edge_edge* ee_records_dev, void* stream);

/* ---- batches: many scenes certified in one launch ------------------------ */
/* One scene of a batch: its geometry (scene-local indices) and object ids,
 * its candidate pair buffers and counts (written by p2c_batch_candidates or
 * p2c_scene_candidates) and where its certificates go.  An array of these
 * lives in device memory (and, for p2c_batch_candidates, a host copy). */
typedef struct p2c_batch_scene {
  const double* v_t0;              /* nv x 3 */
  const double* v_t1;              /* nv x 3 */
  const int32_t* faces;            /* nf x 3 */
  const int32_t* edges;            /* ne x 2 */
  uint64_t* vf_pairs;              /* vf_cap entries */
  uint64_t* ee_pairs;              /* ee_cap entries */
  int64_t vf_cap, ee_cap;
  uint64_t* counts;                /* 4 entries, as p2c_scene_candidates writes them */
  p2c_interval_result* vf_results; /* vf_cap entries */
  p2c_interval_result* ee_results; /* ee_cap entries */
  const int32_t* v_obj;            /* nv object ids (< 0: vertex in no face) */
  const int32_t* f_obj;            /* nf */
  const int32_t* e_obj;            /* ne */
  int64_t nv, nf, ne;
  double thickness;
  int32_t exclude_self;
  int32_t n_obj;
} p2c_batch_scene;

/* Workspace of p2c_batch_candidates for the scenes of a host table. */
size_t p2c_batch_candidates_workspace_bytes(const p2c_batch_scene* scenes_host, int32_t n_scenes);

/* Swept-AABB candidates of every scene of a batch in one launch sequence
 * (about 35 launches whatever the number of scenes): the algorithm of
 * p2c_scene_candidates with scene-segmented reductions, one radix sort of
 * (scene, list, column, quantised minimum) keys over all primitives, per
 * scene column grids and sweeps that stay inside their scene, then one sort
 * of all scenes' pairs.  Each scene's pairs are written sorted and padded
 * with ~0 up to its capacity (the order p2c_scene_candidates with
 * sort_pairs = 1 writes) and its counts as p2c_scene_candidates writes them.
 * scenes_host is read on the host for the sizes (nv, nf, ne, caps); the
 * kernels read scenes_dev (the same table in device memory).  Every scene
 * needs nv, nf, ne < 2^22. */
int p2c_batch_candidates(const p2c_batch_scene* scenes_host, const p2c_batch_scene* scenes_dev, int32_t n_scenes,
                         void* workspace_dev, size_t workspace_bytes, void* stream);

/* Launch shape of the batch certifier (the autotuned parameters). */
typedef struct p2c_batch_tuning {
  int32_t blocks_per_sm;  /* resident blocks of 4 warps per SM; 0: the occupancy maximum */
  int32_t fetch_limit;    /* queries a warp holds at once (1..32); 0: from the batch size */
  int32_t helper_warps;   /* idle warps that stay for exported subtrees; 0: 2 per SM */
  int32_t reserved;
} p2c_batch_tuning;

size_t p2c_batch_certify_workspace_bytes(int32_t n_scenes);

/* Certificates of every candidate pair of every scene of a batch in ONE
 * persistent launch: the scenes' VF lists then EE lists form two global
 * queues that all warps drain together, so small and large scenes share the
 * GPU.  Per scene, summaries_dev[s] (may be NULL) receives the
 * CertificateEngine::Evaluate reduction exactly as p2c_scene_certify writes
 * it; undecided candidates of all scenes are appended to the one queue
 * undecided_queue_dev (may be NULL), in completion order, as
 * (scene << 40 | (family - 1) << 39 | pair position): slots come from one
 * launch-wide counter, summaries_dev[s].undecided_queued counts scene s's
 * entries, and the queue holds the first min(sum, undecided_cap) of them.  A
 * scene with an entry past the capacity gets bit 8 in its summary's error
 * word.  No host sync; the sizes are read on the device.  tuning may be NULL
 * (defaults). */
int p2c_batch_certify(const p2c_batch_scene* scenes_dev, int32_t n_scenes, double interval_t0, double interval_t1,
                      const p2c_cert_config* config, uint32_t family_mask, p2c_scene_summary* summaries_dev,
                      uint64_t* undecided_queue_dev, int64_t undecided_cap, const p2c_batch_tuning* tuning,
                      void* workspace_dev, size_t workspace_bytes, void* stream);

/* ---- candidate groups: scheduled any-hit with fallback replay ------------ */
/* Per-call totals of p2c_group_anyhit. */
typedef struct p2c_anyhit_summary {
  uint64_t candidates;          /* candidates considered: min(*count_dev, cap) */
  uint64_t groups;              /* groups with at least one candidate */
  uint64_t detected_groups;     /* groups with a hit (each group stops at its first hit) */
  uint64_t proposal_calls;      /* certificates the proposal phase counts */
  uint64_t fallback_calls;      /* certificates the fallback replay counts */
  uint64_t fallback_groups;     /* groups with no hit among their proposals */
  uint64_t first_hit_rank_sum;  /* over detected groups: calls up to and including the hit */
  uint64_t speculative;         /* certificates computed on the device and discarded
                                   (started before an earlier candidate of their group hit) */
  uint64_t error_word;          /* 1: time budget, 4: non-finite geometry (counted as a hit),
                                   8: object id outside [0, n_obj) or pair index outside the
                                   scene (the candidate is left out), 16: NaN score (ranked last) */
} p2c_anyhit_summary;

/* Workspace of p2c_group_anyhit for cap candidates and n_obj objects. */
size_t p2c_group_anyhit_workspace_bytes(int64_t cap, int32_t n_obj);

/* Scheduled any-hit over one family's candidate pairs of a scene, with
 * conservative fallback replay: the scene tool's RunScheduledAnyHitRows
 * (tools/scene_object_envelope_native_ti_walltime.cpp:1283-1410) with the
 * reference certifier as the exact judge (hit = collision or undecided).
 *   - group of a candidate = unordered object pair (GroupKey :756-770),
 *     index lo * n_obj + hi with the scene's v_obj/f_obj (family 1) or e_obj
 *     (family 2);
 *   - proposals: per group the top_k candidates by score, higher first,
 *     certified in that order until the first hit;
 *   - fallback replay: every other candidate of a group without a proposal
 *     hit, in candidate order, until the first hit.
 * Ties in score rank the lower candidate index first (the reference's heap
 * order is unspecified for ties; with distinct scores both orders agree).
 * The device certifies candidates speculatively in parallel and cancels those
 * behind a known hit; the reported calls, hits and groups are exactly the
 * sequential procedure's.  n = min(*count_dev, cap) is read on the device, so
 * this can follow p2c_scene_candidates without a host sync.  Outputs (each
 * optional): evaluated_dev[n] (0: not called, 1: proposal call, 2: fallback
 * call), hit_dev[n] (1: called and hit), per group (n_obj * n_obj) detected,
 * proposal calls and fallback calls, and the summary. */
int p2c_group_anyhit(const p2c_scene* scene, int family, const uint64_t* pairs_dev, int64_t cap,
                     const uint64_t* count_dev, const double* scores_dev, int64_t top_k,
                     double interval_t0, double interval_t1, const p2c_cert_config* config,
                     uint8_t* evaluated_dev, uint8_t* hit_dev, uint8_t* group_detected_dev,
                     int64_t* group_proposal_calls_dev, int64_t* group_fallback_calls_dev,
                     p2c_anyhit_summary* summary_dev, void* workspace_dev, size_t workspace_bytes,
                     void* stream);

/* The seeded scheduler stub: scores_dev[i] = a uniform score in [0, 1) of
 * (seed, family, pairs_dev[i]) for i < min(*count_dev, cap) (count_dev may be
 * NULL: all cap entries), 0 beyond.  A score depends only on the candidate's
 * identity (family and pair key), so a candidate is ranked the same alone and
 * in any batch.  It stands in for the learned scheduler's output (the
 * reference tool's "random" policy, ScoreCandidate
 * tools/scene_object_envelope_native_ti_walltime.cpp:1102-1106, plays the
 * same role); callers with a scheduler pass its scores instead. */
int p2c_stub_scores(const uint64_t* pairs_dev, const uint64_t* count_dev, int64_t cap, int family, uint64_t seed,
                    double* scores_dev, void* stream);

/* Workspace of p2c_batch_anyhit for the scenes of a host table. */
size_t p2c_batch_anyhit_workspace_bytes(const p2c_batch_scene* scenes_host, int32_t n_scenes, uint32_t family_mask);

/* p2c_group_anyhit for every (scene, family) of a batch in one launch
 * sequence (about twenty launches whatever the number of scenes): groups are
 * the object pairs of one scene and one family, so every scene gets exactly
 * what p2c_group_anyhit gives it alone with the same scores and top_k.
 * Candidates are each scene's first min(counts[f], cap) pairs (read on the
 * device, so this can follow p2c_batch_candidates without a host sync).
 * Scores: scores_dev (device array of 2 * n_scenes device pointers, entry
 * 2 * s + family - 1 positional over that list's capacity), or, when NULL,
 * the scheduler stub of p2c_stub_scores with seed seeds_dev[s] (seeds_dev
 * NULL: seed 0).  Outputs (each optional): summaries_dev[2 * s + family - 1]
 * (p2c_anyhit_summary of that scene and family); group_detected_dev, one byte
 * per group, and evaluated_dev / hit_dev, one byte per candidate slot, in the
 * batch's index spaces (family-major, then scene: segment k = (family - 1) *
 * n_scenes + s holds that list's capacity of candidate slots and n_obj^2
 * groups).  scenes_host is read on the host for sizes (caps, n_obj). */
int p2c_batch_anyhit(const p2c_batch_scene* scenes_host, const p2c_batch_scene* scenes_dev, int32_t n_scenes,
                     uint32_t family_mask, const double* const* scores_dev, const uint64_t* seeds_dev, int64_t top_k,
                     double interval_t0, double interval_t1, const p2c_cert_config* config,
                     p2c_anyhit_summary* summaries_dev, uint8_t* group_detected_dev, uint8_t* evaluated_dev,
                     uint8_t* hit_dev, void* workspace_dev, size_t workspace_bytes, void* stream);

/* ---- serving: continuous batching of CCD steps on one GPU ---------------- */
/* A server keeps registered meshes (topology, object ids) resident on its
 * device together with their candidate state (pair capacities fitted to the
 * last step), and one device arena of memory_budget bytes allocated at
 * creation.  Requests are CCD steps of a registered mesh (the vertex
 * trajectories of one step, host memory).  p2c_serve_poll retires finished
 * groups and admits waiting requests, in admission order, into free slots:
 * the requests admitted together (up to max_group, and up to 600,000
 * triangles unless one request alone is larger) form a group on the slot's
 * own stream
 * (trajectories in; candidates of every request in one p2c_batch_candidates
 * sequence; then either the certificates of every candidate, one
 * p2c_batch_certify launch, or the scheduled any-hit with fallback replay of
 * every request, one p2c_batch_anyhit sequence; summaries out), as long as
 * the group's memory fits a free range of the arena.  Groups on different
 * slots overlap on the device.  A request whose candidates outgrew its
 * buffers (or, certifying every candidate, the undecided queue) is re-run
 * with larger ones, so every result is the complete answer for its step: the
 * one the step gets alone.  The reference has no serving layer; the
 * ownership model of each step is RunCudaBatch's (certificate_cuda.cu:456-552:
 * host arrays in, host results out) with device memory held across steps.
 * One host thread drives a server (the calls are not re-entrant). */
#define P2C_SERVE_CERTIFY 0  /* certificates of every candidate */
#define P2C_SERVE_ANYHIT 1   /* scheduled any-hit with fallback replay per object-pair group */

typedef struct p2c_serve_config {
  int32_t slots;              /* groups in flight (one CUDA stream each), >= 1 */
  int32_t max_group;          /* requests admitted into one group, >= 1 */
  int32_t narrow;             /* P2C_SERVE_CERTIFY or P2C_SERVE_ANYHIT */
  int32_t top_k;              /* any-hit proposals per group (RunScheduledAnyHitRows' proposal_top_k) */
  int64_t memory_budget;      /* device arena bytes; 0: half the free device memory at creation */
  int64_t undecided_capacity; /* first size of a group's undecided queue (certify mode), grows on overflow */
  p2c_cert_config cert;       /* CertificateEngineConfig of every certificate */
  double interval_t0, interval_t1;
} p2c_serve_config;

typedef struct p2c_serve p2c_serve;  /* opaque */

/* A mesh: host arrays copied to the device at registration. */
typedef struct p2c_serve_mesh {
  const int32_t* faces;  /* nf x 3 */
  const int32_t* edges;  /* ne x 2 */
  const int32_t* v_obj;  /* nv */
  const int32_t* f_obj;  /* nf */
  const int32_t* e_obj;  /* ne */
  int64_t nv, nf, ne;
  int32_t n_obj;          /* object ids < n_obj; candidate groups are object pairs */
  int32_t exclude_self;   /* 1: no candidates between primitives of one object */
  double thickness;
  int64_t vf_capacity, ee_capacity;  /* first pair capacities (0: from the face count) */
} p2c_serve_mesh;

/* A CCD step.  v_t0 / v_t1 (nv x 3 doubles, host memory; page-locked memory
 * lets the copies overlap) must stay valid until the request's result is
 * returned.  Optional host outputs, filled before the result is returned:
 * vf_results / ee_results (certify mode: the certificates of the first
 * results_cap candidates of each list), undecided (certify mode: (family -
 * 1) << 63 | pair position of each undecided certificate, the fallback-replay
 * list, up to undecided_cap entries), group_detected (any-hit mode: n_obj^2
 * bytes for the VF groups then n_obj^2 for the EE groups, index lo * n_obj +
 * hi, up to groups_cap bytes).  seed is the scheduler stub's seed (any-hit). */
typedef struct p2c_serve_request {
  int32_t mesh_id;
  int32_t pad;
  const double* v_t0;
  const double* v_t1;
  uint64_t seed;
  p2c_interval_result* vf_results;
  p2c_interval_result* ee_results;
  int64_t results_cap;
  uint64_t* undecided;
  int64_t undecided_cap;
  uint8_t* group_detected;
  int64_t groups_cap;
} p2c_serve_request;

typedef struct p2c_serve_result {
  int64_t request_id;
  int32_t status;        /* P2C_OK, or the error code that failed this request (p2c_last_error) */
  int32_t reruns;        /* re-runs after a buffer overflow */
  double latency_ms;     /* device clock: admission to the completion of its group */
  uint64_t vf_candidates, ee_candidates;
  uint64_t undecided_entries;        /* certify mode: entries of its fallback-replay list */
  uint64_t truncated;                /* bits: 1 results, 2 undecided list, 4 group decisions beyond the caps */
  p2c_scene_summary certify;         /* certify mode: the Evaluate reduction of its candidates */
  p2c_anyhit_summary anyhit[2];      /* any-hit mode: VF and EE summaries */
} p2c_serve_result;

typedef struct p2c_serve_stats {
  uint64_t admitted, completed, failed, groups, reruns;
  uint64_t pending, in_flight;
  uint64_t candidates;       /* candidates of completed requests */
  uint64_t calls;            /* certificates the procedure called (certify: all candidates) */
  uint64_t arena_bytes, arena_in_use, arena_peak;
} p2c_serve_stats;

/* Create a server on the current device (allocates its arena, streams and
 * events); *out receives the handle. */
int p2c_serve_create(const p2c_serve_config* config, p2c_serve** out);
/* Wait for groups in flight, then free everything the server holds. */
int p2c_serve_destroy(p2c_serve* server);
/* Copy a mesh to the device; *mesh_id receives its id. */
int p2c_serve_register_mesh(p2c_serve* server, const p2c_serve_mesh* mesh, int32_t* mesh_id);
/* A request arrives: it waits for admission (the next poll).  Its arrival is
 * stamped on the device clock now; *request_id receives its id. */
int p2c_serve_admit(p2c_serve* server, const p2c_serve_request* request, int64_t* request_id);
/* Retire finished groups, launch waiting requests into free slots, and
 * return up to max_results finished requests (the rest at later polls). */
int p2c_serve_poll(p2c_serve* server, p2c_serve_result* results, int32_t max_results, int32_t* n_results);
int p2c_serve_read_stats(p2c_serve* server, p2c_serve_stats* stats);

/* ---- proxy scenes: patch-level candidates with time slabs ---------------- */
/* The proxy primitives of a built ProxyScene (rt_candidate/proxy_scene.h:29-46)
 * as device arrays; proxy i has proxy_id i. */
typedef struct p2c_proxy_scene {
  uint64_t query_id;
  int64_t n;                     /* proxy primitives */
  const uint32_t* object_id;
  const uint32_t* patch_id;
  const uint32_t* slab_id;
  const uint8_t* proxy_type;     /* 1 swept AABB, 2 capsule */
  const double* t0;              /* slab interval */
  const double* t1;
  const double* bounds;          /* n x 6: min x, y, z, max x, y, z */
  const double* motion_bound;    /* n x 4: translation_bound, rotation_angle, radial_motion_bound,
                                    conservative_radius */
  /* Optional widths of the ids (0 = up to 32 bits): every slab id < 2^slab_bits, object id <
   * 2^object_bits, patch id < 2^patch_bits.  Narrower sort keys; an id outside its width sets
   * bit 8 of the error word and the results are void (run again without the hint). */
  uint32_t slab_bits, object_bits, patch_bits;
  uint32_t pad0;
} p2c_proxy_scene;

/* RawCandidateHit (rt_candidate/candidate_buffer.h:19-31), 64 bytes. */
typedef struct p2c_raw_candidate_hit {
  uint64_t query_id;
  uint64_t pair_key;             /* lo << 32 | hi proxy index */
  uint32_t proxy_a_index, proxy_b_index;
  uint32_t slab_id;
  uint32_t rt_hit_count;
  uint32_t flags;                /* 1 valid | 2 AABB overlap */
  uint32_t reserved0;
  float motion_bound[4];
  uint32_t reserved1, reserved2;
} p2c_raw_candidate_hit;

/* CandidateRecord (common/runtime_contracts.h:41-56), 80 bytes. */
typedef struct p2c_candidate_record {
  uint32_t schema_version;
  uint32_t pad0;
  uint64_t candidate_id;
  uint64_t query_id;
  uint32_t slab_id;
  uint32_t object_a_id, patch_a_id, object_b_id, patch_b_id;
  uint8_t proxy_type_a, proxy_type_b;
  uint8_t pad1[2];
  uint32_t rt_hit_count;
  float motion_bound[4];
  uint32_t proxy_features_offset;
  uint32_t flags;
  uint32_t pad2;
} p2c_candidate_record;

/* Workspace of p2c_proxy_candidates for n proxies, raw_cap hits and the
 * scene's slab_bits hint (0: none; a hint of at most 6 bits adds a direct
 * (slab, column) table of 2^(slab_bits + 14) x 16 bytes). */
size_t p2c_proxy_candidates_workspace_bytes(int64_t n_proxies, int64_t raw_cap, uint32_t slab_bits);

/* Candidates of a proxy scene: GenerateRawCandidatesCpu then
 * CompactRawCandidates (rt_candidate/candidate_buffer.cpp:144-227) on the
 * device.  Raw hits are the proxy pairs of different objects in one slab
 * whose time intervals and inclusive AABBs overlap, written in the
 * reference's (i, j) order; candidates are the hits compacted by (slab,
 * first (object, patch), second (object, patch), proxy types) with the first
 * proxy the smaller (object, patch, proxy) tuple, in that key order, with
 * candidate_id 1, 2, ..., hit counts summed, motion bounds maxed and flags
 * or-ed.  counts_dev[0..2] = {raw hits, candidates, error word (1: a proxy
 * fails ValidateProxyScene's per-proxy checks, rt_candidate/proxy_scene.cpp:
 * 143-151: type, finite t0 < t1, finite ordered bounds; 2: a hit's float
 * motion bound is negative or non-finite, which ValidateRawHit rejects in
 * compaction, candidate_buffer.cpp:95-99; 4: raw_cap overflowed; 8: an id
 * outside its width hint)}.  Proxy
 * ids equal to the array index and the global slab partition (:58-85) are
 * the caller's checks.  Raw hits beyond raw_cap are dropped (the count is
 * the total); candidate capacity is raw_cap; raw_cap 0 only counts.  No host
 * sync. */
int p2c_proxy_candidates(const p2c_proxy_scene* scene, p2c_raw_candidate_hit* raw_dev, int64_t raw_cap,
                         p2c_candidate_record* candidates_dev, uint64_t* counts_dev, void* workspace_dev,
                         size_t workspace_bytes, void* stream);

/* Workspace of p2c_compact_raw_candidates (as p2c_proxy_candidates with
 * raw_cap = n_raw). */
size_t p2c_compact_raw_candidates_workspace_bytes(int64_t n_proxies, int64_t n_raw, uint32_t slab_bits);

/* CompactRawCandidates (rt_candidate/candidate_buffer.cpp:181-227) on n_raw
 * given hits of a proxy scene (from any tracer): each hit checked as
 * ValidateRawHit does (:71-101), then the same compaction, order and ids as
 * p2c_proxy_candidates.  candidates_dev holds n_raw records.
 * counts_dev[0..3] = {n_raw, candidates, error word (1: a proxy fails the
 * per-proxy checks; 16: a candidate's summed rt_hit_count overflows 32
 * bits), the first invalid hit as (hit index << 4 | check) or ~0: check 1 not
 * marked valid, 2 zero query id, 3 query id differs from the scene's, 4 proxy
 * index out of range, 5 the same proxy twice, 6 pair_key mismatch, 7 one
 * object, 8 slab mismatch, 9 motion bound negative or non-finite}.  With an
 * invalid hit the records are meaningless.  No host sync. */
int p2c_compact_raw_candidates(const p2c_proxy_scene* scene, const p2c_raw_candidate_hit* raw_dev, int64_t n_raw,
                               p2c_candidate_record* candidates_dev, uint64_t* counts_dev, void* workspace_dev,
                               size_t workspace_bytes, void* stream);

/* ---- proxy scene build: patches x motion segments x time slabs --------------- */
/* MotionSegment (geometry/motion.h:14-19): a rigid motion from pose_t0 at t0 to
 * pose_t1 at t1; rotation quaternions are x, y, z, w. */
typedef struct p2c_motion_segment {
  double t0, t1;
  double translation_t0[3];
  double rotation_t0[4];
  double translation_t1[3];
  double rotation_t1[4];
} p2c_motion_segment;

/* ProxyObjectBuildInput (rt_candidate/proxy_scene.h:15-22).  Its patches are
 * entries [patch_offset, patch_offset + n_patches) of the device patch
 * arrays; its motion segments are a HOST array. */
typedef struct p2c_proxy_object_input {
  uint32_t object_id;
  uint32_t proxy_type;               /* 1 swept AABB, 2 capsule */
  uint32_t slabs_per_motion_segment;
  uint32_t pad0;
  double eps_proxy;
  int64_t patch_offset, n_patches;
  int64_t n_segments;
  const p2c_motion_segment* segments; /* host */
} p2c_proxy_object_input;

/* Device outputs of p2c_proxy_scene_build, n proxies each (the inputs of
 * p2c_proxy_candidates plus the rest of ProxyPrimitive).  motion_detail and
 * capsule_radius may be NULL. */
typedef struct p2c_proxy_build_out {
  uint32_t* object_id;
  uint32_t* patch_id;
  uint32_t* slab_id;
  uint32_t* motion_segment_id;
  uint8_t* proxy_type;
  double* t0;
  double* t1;
  double* bounds;          /* n x 6 */
  double* motion_bound;    /* n x 4: translation_bound, rotation_angle, radial_motion_bound,
                              conservative_radius */
  double* motion_detail;   /* n x 8: center_t0 xyz, center_t1 xyz, center_rotation_bound,
                              surface_rotation_bound */
  double* capsule_radius;  /* n: the inflated radius of a capsule proxy, 0 for a swept AABB */
} p2c_proxy_build_out;

/* Proxies the objects expand to (sum of segments x slabs x patches), after
 * the per-object checks of BuildProxyScene; -1 and the last error on an
 * invalid input. */
int64_t p2c_proxy_scene_count(const p2c_proxy_object_input* objects, int64_t n_objects);
size_t p2c_proxy_scene_build_workspace_bytes(const p2c_proxy_object_input* objects, int64_t n_objects);

/* BuildProxyScene (rt_candidate/proxy_scene.cpp:156-213): for each object,
 * motion segment, uniform time slab and patch (in that order) one proxy with
 * the patch's motion bound over the slab (ComputePatchMotionBound,
 * geometry/motion_utils.cpp:269-325) and its swept-AABB or capsule bounds
 * inflated by eps_proxy (geometry/proxy.cpp:70-131).  The rigid pose of each
 * (object, segment, slab) end is computed on the host with the C library's
 * acos/sin/cos, as the reference does; the per-patch transforms and bounds,
 * all additions, products, quotients and square roots, run on the device.
 * Object, segment and slab checks and the global slab partition
 * (proxy_scene.cpp:58-85) fail the call with the reference's message;
 * per-patch failures set bits of *error_word_dev (1 patch centre non-finite,
 * 2 patch radius negative or non-finite, 4 swept AABB invalid before
 * inflation, 8 capsule radius invalid, 16 final bounds invalid).
 * Every object's patch range must lie inside the n_patch_entries patch
 * entries.  proxy_cap must be at least p2c_proxy_scene_count.  No host sync. */
int p2c_proxy_scene_build(uint64_t query_id, const p2c_proxy_object_input* objects, int64_t n_objects,
                          const uint32_t* patch_id_dev, const double* patch_center_dev,
                          const double* patch_radius_dev, int64_t n_patch_entries, int64_t proxy_cap,
                          const p2c_proxy_build_out* out,
                          uint64_t* error_word_dev, void* workspace_dev, size_t workspace_bytes, void* stream);

/* ---- proposal feature rows (the learned scheduler's inputs) -------------- */
/* CandidateDensityStats (rt_candidate/candidate_generation_result.h:21-37)
 * without its timing and backend name, 96 bytes. */
typedef struct p2c_candidate_density {
  uint64_t query_id;
  uint64_t proxy_count, object_count, slab_count, cross_object_same_slab_pair_count;
  uint64_t raw_hit_count, compact_candidate_count;
  double raw_hits_per_proxy, candidates_per_proxy, candidates_per_slab, aabb_overlap_ratio;
  double avg_rt_hits_per_candidate;
} p2c_candidate_density;

/* ProposalFeatureRow (proposal/proposal_features.h:27-43), 256 bytes. */
typedef struct p2c_proposal_feature_row {
  uint32_t schema_version;
  uint32_t pad0;
  uint64_t query_id;
  uint64_t candidate_id;
  uint32_t slab_id;
  uint32_t object_a_id, patch_a_id, object_b_id, patch_b_id;
  float features[32];
  float interval_targets[8];
  float family_targets[8];
  float priority_target, cost_target, uncertainty_target;
  uint32_t target_mask;
  uint32_t pad1;
} p2c_proposal_feature_row;

size_t p2c_proposal_feature_rows_workspace_bytes(int64_t n_proxies);

/* The density stats and proposal feature rows of a proxy scene's candidates,
 * on the device: ComputeCandidateDensityStats (rt_candidate/
 * candidate_stats.cpp:128-170) into *density_dev and ExtractProposalFeatureRows
 * (proposal/proposal_features.cpp:236-259, rows by FillFeatureRow :122-205)
 * into rows_dev[0 .. min(counts_dev[1], cap)).  counts_dev and candidates_dev
 * are p2c_proxy_candidates' outputs for the same scene (no host sync between
 * the calls).  Each candidate side maps to the first proxy in scene order with
 * its (slab, object, patch, type).  *error_word_dev: bit 1 a candidate fails
 * ValidateCandidateRecord (common/validators.cpp:160-181), bit 2 a candidate
 * side maps to no proxy; such rows are zero; bit 4 a proxy id beyond its
 * width hint (results void; p2c_proxy_candidates flags the same scene).  The
 * scene's id width hints narrow the sorts, and when all three are set and
 * slab, type, object and patch fit one 64-bit word the first-proxy lookup is
 * one sort and one binary search per side.  No host sync. */
int p2c_proposal_feature_rows(const p2c_proxy_scene* scene, const p2c_candidate_record* candidates_dev,
                              int64_t cap, const uint64_t* counts_dev, p2c_candidate_density* density_dev,
                              p2c_proposal_feature_row* rows_dev, uint64_t* error_word_dev, void* workspace_dev,
                              size_t workspace_bytes, void* stream);

/* BuildProposalFeatureRowsFromRuntimeCandidates (proposal/
 * proposal_policy.cpp:568-592, rows by :184-226): rows from n candidate
 * records alone, the density ratios of primitive_count / raw_hit_count /
 * compact_candidate_count (MakeRuntimeDensityDerivedStats :44-58) and each
 * query's conservative family mask (n_masks query ids in ascending order with
 * their masks; a query absent or with mask 0 gets both families).  Bit 1 of
 * *error_word_dev: a candidate fails ValidateCandidateRecord (its row is
 * zero).  primitive_count 0 fails the call with the reference's message.  No
 * host sync. */
int p2c_runtime_feature_rows(const p2c_candidate_record* candidates_dev, int64_t n, uint64_t primitive_count,
                             uint64_t raw_hit_count, uint64_t compact_candidate_count,
                             const uint64_t* mask_query_ids_dev, const uint32_t* masks_dev, int64_t n_masks,
                             p2c_proposal_feature_row* rows_dev, uint64_t* error_word_dev, void* stream);

/* ---- audit rows of an exact work queue ------------------------------------- */
/* The ExactWorkItem fields (common/runtime_contracts.h:67-81) an audit row
 * reads, 56 bytes; candidate_id is the item's parent_candidate_id. */
typedef struct p2c_audit_item {
  uint64_t query_id, candidate_id, work_item_id;
  double interval_t0, interval_t1;
  float priority_score;
  uint32_t feature_family_mask;
  uint16_t depth;
  uint16_t pad[3];
} p2c_audit_item;

/* AuditLogRow (common/runtime_contracts.h:101-114), 80 bytes. */
typedef struct p2c_audit_row {
  uint64_t event_id, query_id, candidate_id, work_item_id;
  uint8_t stage;                 /* AuditStage: 2 exact (dequeue), 4 certify */
  uint8_t pad0;
  uint16_t action;               /* 1 dequeued, 2 collision, 3 separation, 4 undecided, 5 invalid input */
  uint16_t depth;
  uint16_t pad1;
  double interval_t0, interval_t1;
  uint64_t timestamp_us;
  double aux_value0, aux_value1;
} p2c_audit_row;

/* The audit log ProcessExactWorkQueueCpu (certificate/certificate_engine.cpp:
 * 593-661) writes for n certified work items, from their certificates on the
 * device (p2c_certify_queries' output): per item, with emit_dequeue_events a
 * dequeue row (stage exact, action dequeued, aux = priority score, family
 * mask), then a certify row (stage certify, action from the status and
 * reason code, aux = safe_margin_lb for a separation else toi_upper, and the
 * next refinement mode); event ids and timestamps count up from
 * first_event_id / first_timestamp_us in that order (rows_dev holds n x 2 or
 * n rows).  error_dev[0] bit 1: a row fails ValidateAuditLogRow
 * (common/validators.cpp:295-315), error_dev[1] the first such row.  No host
 * sync. */
int p2c_audit_rows(const p2c_audit_item* items_dev, const p2c_query_certificate* certs_dev, int64_t n,
                   uint64_t first_event_id, uint64_t first_timestamp_us, int emit_dequeue_events,
                   p2c_audit_row* rows_dev, uint64_t* error_dev, void* stream);

/* ---- runtime exact work queue from proposals ------------------------------- */
/* ProposalOutput (common/runtime_contracts.h:58-65), 88 bytes. */
typedef struct p2c_proposal_output {
  uint64_t candidate_id;
  float interval_scores[8];
  float family_scores[8];
  float priority_score, cost_score, uncertainty_score;
  uint32_t pad0;
} p2c_proposal_output;

/* ExactWorkItem (common/runtime_contracts.h:67-81), 80 bytes. */
typedef struct p2c_exact_work_item {
  uint64_t work_item_id, parent_candidate_id, query_id;
  uint32_t slab_id, patch_a_id, patch_b_id, pad0;
  double interval_t0, interval_t1;
  uint32_t feature_family_mask, topk_feature_ids_offset;
  uint16_t depth;
  uint16_t pad1;
  float priority_score;
  uint8_t source;                /* ProposalSource: 0 raw, 1 refined, 2 fallback */
  uint8_t pad2[7];
} p2c_exact_work_item;

/* ProposalSchedulingConfig (proposal/proposal_policy.h:13-23). */
typedef struct p2c_scheduling_config {
  uint64_t first_work_item_id;
  uint32_t conservative_feature_family_mask;
  uint32_t preserve_candidate_order;
  double fallback_interval_t0, fallback_interval_t1;
  float family_score_threshold, uncertainty_fallback_threshold, ood_abs_feature_threshold;
  uint32_t pad0;
} p2c_scheduling_config;

/* ProposalScheduleStats (proposal/proposal_policy.h:25-36); monotonic_safe 0/1. */
typedef struct p2c_schedule_stats {
  uint64_t raw_candidate_count, proposal_output_count, work_item_count, fallback_count;
  uint64_t missing_proposal_fallback_count, invalid_proposal_fallback_count, ood_fallback_count;
  uint64_t high_uncertainty_fallback_count, reordered_count, monotonic_safe;
} p2c_schedule_stats;

size_t p2c_schedule_work_items_workspace_bytes(int64_t n_candidates, int64_t n_rows, int64_t n_outputs);

/* The ordered exact work queue from proposals.  mode 0:
 * ScheduleRuntimeExactWorkItemsFromProposals (proposal/proposal_policy.cpp:
 * 595-742): per candidate its feature row and proposal output found by
 * candidate id; mode 1: the binding's aligned-array form (bindings/
 * py_module.cpp:1088-1174): rows and outputs at the same position, the
 * candidate fields from the row and a fallback priority of features[3].  A
 * candidate falls back (conservative family mask, rt-hit priority, source
 * fallback) on a missing, invalid, out-of-distribution or high-uncertainty
 * proposal; otherwise it takes the predicted families and the proposal's
 * priority (source refined).  Unless preserve_candidate_order, the queue is
 * stable-sorted by priority, descending; work item ids count up from
 * first_work_item_id in queue order.  The config is checked on the host
 * (the reference's messages); *error_dev bits: 1 a candidate fails
 * ValidateCandidateRecord, 2 a row id is zero or repeated, 4 an output id is
 * zero or repeated, 8 repeated candidate ids, 16 a work item fails
 * ValidateExactWorkItem, 32 a work item has no exact family, 64 unknown
 * family bits (mode 0), 128 aligned arrays out of candidate order (mode 1);
 * error_dev[1] / [2]: the first queue position with no family / with unknown
 * bits (~0 if none; the reference reports the earlier one).  Family masks per
 * query: n_masks ascending query ids with their masks.  No host sync. */
int p2c_schedule_work_items(int mode, const p2c_candidate_record* candidates_dev, int64_t n_candidates,
                            const p2c_proposal_feature_row* rows_dev, int64_t n_rows,
                            const p2c_proposal_output* outputs_dev, int64_t n_outputs,
                            const uint64_t* mask_query_ids_dev, const uint32_t* masks_dev, int64_t n_masks,
                            const p2c_scheduling_config* config, p2c_exact_work_item* items_dev,
                            p2c_schedule_stats* stats_dev, uint64_t* error_dev, void* workspace_dev,
                            size_t workspace_bytes, void* stream);

/* RunDummyProposalScheduleFromRuntimeCandidates (cpp/proposal/
 * proposal_policy.cpp:744-858; binding py_module.cpp:1009-1033) for n device
 * candidates (bypass == 0): the density-derived dummy proposals, the
 * out-of-distribution fallback, a stable sort by priority (unless the config
 * preserves candidate order) and the checks.  With rows_dev and outputs_dev
 * non-NULL the artifacts are materialized too (rows as
 * p2c_runtime_feature_rows; outputs from them).  bypass != 0 is the raw
 * queue of GenerateExternalBatchDummyProposalScheduleOrThrow
 * (py_module.cpp:290-318): one kRaw item per candidate in order, its query's
 * mask, priority rt_hit_count, no config check.  Workspace:
 * p2c_schedule_work_items_workspace_bytes(n, 0, 0).  error_dev[0] as for
 * p2c_schedule_work_items (bits 1 and 16).  No host sync. */
int p2c_dummy_schedule(int bypass, const p2c_candidate_record* candidates_dev, int64_t n, uint64_t primitive_count,
                       uint64_t raw_hit_count, uint64_t compact_candidate_count, const uint64_t* mask_query_ids_dev,
                       const uint32_t* masks_dev, int64_t n_masks, const p2c_scheduling_config* config,
                       p2c_proposal_feature_row* rows_dev, p2c_proposal_output* outputs_dev,
                       p2c_exact_work_item* items_dev, p2c_schedule_stats* stats_dev, uint64_t* error_dev,
                       void* workspace_dev, size_t workspace_bytes, void* stream);

/* ---- candidate-group early-stop replay ----------------------------------- */
/* DenseGroupEarlyStopConfig (cpp/common/group_scheduler.h:24-29) plus the
 * width of the query ids (bits above it must be zero; 0 = 64). */
typedef struct p2c_dense_group_config {
  float uncertainty_fallback_threshold;
  uint32_t representative_attempt_limit;
  double interval_miss_penalty_scale;
  int32_t preserve_input_order;
  int32_t query_bits;
} p2c_dense_group_config;

/* DenseGroupEarlyStopStats (group_scheduler.h:31-61) without the host
 * timings, and the first invalid row: error_kind 1 a zero query or candidate
 * id, 2 a non-finite field (group_scheduler.cpp:81-88), at row error_row
 * (-1 none; the totals are then meaningless). */
typedef struct p2c_dense_group_stats {
  uint64_t candidate_count;
  uint64_t group_count;
  uint64_t positive_group_count;
  uint64_t no_proposal_exact_calls;
  double no_proposal_exact_work;
  uint64_t learned_exact_calls;
  uint64_t learned_fallback_calls;
  uint64_t learned_interval_hit_count;
  uint64_t learned_interval_miss_count;
  double learned_exact_work;
  double first_positive_rank_sum;
  double cost_before_first_positive_sum;
  uint64_t tp;
  uint64_t tn;
  uint64_t fp;
  uint64_t fn;
  uint64_t reordered_count;
  uint64_t high_uncertainty_group_count;
  int64_t error_row;
  int32_t error_kind;
  int32_t pad;
} p2c_dense_group_stats;

size_t p2c_dense_group_early_stop_workspace_bytes(int64_t n);

/* RunNativeDenseGroupExactEarlyStopOrThrow (cpp/bindings/py_module.cpp:
 * 1179-1311) over RunDenseGroupExactEarlyStop (common/group_scheduler.cpp:
 * 60-239) for n device rows: query_id, candidate_id, cost_target,
 * oracle_trace (n x 8 doubles), interval_scores (n x 8 floats) and the
 * priority, cost and uncertainty scores.  Writes *stats_dev (device); every
 * total, the double ones included, equals the reference's bit for bit.
 * Invalid configurations return P2C_ERR_INVALID with the reference's
 * messages.  No host sync. */
int p2c_dense_group_early_stop(int64_t n, const uint64_t* query_id_dev, const uint64_t* candidate_id_dev,
                               const float* cost_target_dev, const double* oracle_trace_dev,
                               const float* interval_scores_dev, const float* priority_score_dev,
                               const float* cost_score_dev, const float* uncertainty_score_dev,
                               const p2c_dense_group_config* config, p2c_dense_group_stats* stats_dev,
                               void* workspace_dev, size_t workspace_bytes, void* stream);

/* The left-to-right double sum of n non-negative terms (NaN-free; +inf
 * allowed), bit-identical to `s = 0; for (i) s += terms[i];`: the ordered
 * accumulation RunDenseGroupExactEarlyStop makes (group_scheduler.cpp:
 * 128-230), computed with block scans instead of one dependent add per term.
 * Writes *out_dev; one block; no host sync. */
int p2c_ordered_sum(const double* terms_dev, int64_t n, double* out_dev, void* stream);

/* ---- refinement children ------------------------------------------------- */
size_t p2c_refinement_children_workspace_bytes(int64_t n_parents);

/* GenerateConservativeRefinementWorkItems (cpp/certificate/
 * certificate_engine.cpp:663-720) for n_parents work items at once: parent i
 * (interval [parent_t0, parent_t1], depth parent_depth, certificate certs[i])
 * gets at depth < max_child_depth one child [t0, clamp(toi_upper, t0, t1)]
 * for a collision, two halves around 0.5 * (t0 + t1) for an undecided
 * certificate asking for bisection, each only when wider than
 * min_interval_width.  Children are written compacted in parent order
 * (capacity 2 * n_parents): the parent index, interval, depth + 1 and
 * work_item_id first_child_work_item_id + position (the ids of calling the
 * reference once per parent in order with the next free id); the caller
 * copies the parent's other ExactWorkItem fields and sets source = refined.
 * *child_count_dev receives the number written.  A parent whose interval is
 * not 0 <= t0 <= t1 <= 1 gets no child and sets bit 1 of *error_word_dev
 * (may be NULL).  No host sync. */
int p2c_refinement_children(int64_t n_parents, const double* parent_t0_dev, const double* parent_t1_dev,
                            const uint16_t* parent_depth_dev, const p2c_query_certificate* certs_dev,
                            uint16_t max_child_depth, double min_interval_width, uint64_t first_child_work_item_id,
                            int64_t* child_parent_dev, double* child_t0_dev, double* child_t1_dev,
                            uint16_t* child_depth_dev, uint64_t* child_work_item_id_dev, uint64_t* child_count_dev,
                            uint64_t* error_word_dev, void* workspace_dev, size_t workspace_bytes, void* stream);

/* ---- diagnostics ------------------------------------------------------- */
/* FP64 throughput probe: launches independent separately rounded multiply/add
 * chains over a full-occupancy grid and reports the FP64 operations it issues;
 * the caller times it (CUDA events) to obtain the measured FP64 rate that the
 * certifier's roofline is quoted against.  No reference counterpart. */
int p2c_probe_fp64(void* out_dev, int iters, long long* fp64_ops_out, void* stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* P2C_B200_H_ */
