/* RapidBoW-B200: C ABI of the B200-native vocabulary-tree hot path.
 *
 * Every entry point returns an rbw_status (0 = RBW_OK) and never throws; the message of the
 * last failure on the calling thread is available from rbw_last_error().  Handles are opaque.
 * `stream` arguments are cudaStream_t values passed as void* (NULL = legacy default stream).
 * Device buffers are plain device (or managed) pointers; descriptor rows are 128 uint8 bytes
 * and must start on a 16-byte boundary, as the reference requires (vocTreeLookUp.cu:42,71).
 *
 * Each declaration names the reference interface it replaces (file:line in lowsfer/RapidBoW).
 */
#ifndef RAPIDBOW_B200_H
#define RAPIDBOW_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RBW_API __attribute__((visibility("default")))
#else
#define RBW_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    RBW_OK = 0,
    RBW_ERR_INVALID_ARG = 1,   /* std::runtime_error on bad input in the reference */
    RBW_ERR_UNSUPPORTED = 2,   /* the reference prints and returns nullptr (RapidBoW.cpp:37-40) */
    RBW_ERR_OUT_OF_MEMORY = 3,
    RBW_ERR_CUDA = 4,          /* cudaCheck failures */
    RBW_ERR_TIMEOUT = 5,       /* a device-side bounded wait gave up */
    RBW_ERR_INVALID_BLOB = 6,  /* "invalid blob" (Vocabulary.cpp:128-144) */
    RBW_ERR_DUPLICATE = 7,     /* "Duplicate document index" (DataBase.cpp:41-43) */
    RBW_ERR_INTERNAL = 8
} rbw_status;

/* Values match rbow::DataType / rbow::DistanceType (RapidBoW.h:32-48). */
enum { RBW_DATA_BINARY = 0, RBW_DATA_UINT8 = 1 };
enum { RBW_DIST_HAMMING = 0, RBW_DIST_L1 = 1, RBW_DIST_L2 = 2 };
typedef struct {
    int32_t data_type;
    int32_t distance_type;
    uint64_t nb_dims;
} rbw_desc_attr;

/* Initial-center choice for the k-means of every node. */
enum {
    RBW_INIT_REFERENCE = 0, /* the reference's random distinct picks (kmeans.cpp:141-196), default seed */
    RBW_INIT_KMEANSPP = 1,  /* seeded k-means++ over <= 256 sampled members per node */
    RBW_INIT_INJECTED = 2   /* caller-provided descriptor indices per node */
};

/* Build flags.  The reference rounds centers with its --use_fast_math division
 * (kmeans.cu:367); RBW_BUILD_IEEE_DIVISION uses the correctly rounded quotient instead.
 * RBW_BUILD_FLOAT_CENTERS (no counterpart in the reference, whose centers are uint8) keeps fp32
 * centers, c = float(double(sum) / double(count)) of the exact integer sums; distances come from
 * the tensor cores with each center split into hi + lo bf16 parts and fp32 accumulation, and
 * every descriptor whose best-versus-second margin is within the stated error bound is re-scored
 * in FP64 on the GPU, so assignments equal those of an FP64 evaluation (lowest index on ties).
 * Lookups through such a vocabulary use the same arithmetic. */
enum { RBW_BUILD_IEEE_DIVISION = 1, RBW_BUILD_FLOAT_CENTERS = 2 };

/* Center storage of a vocabulary. */
enum { RBW_CENTERS_UINT8 = 0, RBW_CENTERS_FLOAT32 = 1 };

/* Statistics of the build that made a vocabulary (zero for uploaded or deserialised ones). */
typedef struct {
    uint32_t levels;
    uint32_t iterations[16];     /* Lloyd steps run per level */
    double inertia_first[16];    /* float centers: FP64 inertia of the level's first assignment */
    double inertia_last[16];     /*                and of its last one (frozen nodes keep theirs) */
    uint64_t refined[16];        /* float centers: assignments re-scored in FP64, all steps */
    uint64_t assignments[16];    /*                assignments made, all steps */
    double seconds;              /* wall time of the build call */
} rbw_build_stats;

typedef struct {
    uint32_t max_iterations;       /* Lloyd cap; reference: 1000 (kmeans.h:118) */
    uint32_t check_interval;       /* host convergence poll; reference: 4 (kmeans.h:115) */
    uint32_t init_mode;            /* RBW_INIT_* */
    uint32_t flags;                /* RBW_BUILD_* bits */
    uint64_t seed;                 /* RBW_INIT_KMEANSPP */
    const uint32_t* injected_init; /* RBW_INIT_INJECTED: host [levelBeg(L)][B], UINT32_MAX = invalid */
} rbw_build_options;

typedef struct rbw_vocabulary rbw_vocabulary;

/* Lookup algorithms. */
enum {
    RBW_LOOKUP_AUTO = 0,       /* fastest exact path */
    RBW_LOOKUP_TENSOR_U8 = 1,  /* tcgen05 uint8 tensor-core descent with device regroup */
    RBW_LOOKUP_SIMT_F32 = 2,   /* plain FP32 SIMT descent (comparison baseline) */
    RBW_LOOKUP_TENSOR_U8_WARPNODE = 3, /* as TENSOR_U8, the node level of each level pair by warp-level MMAs
                                          in the epilogue warps, so the children MMA need not wait for it */
    RBW_LOOKUP_TENSOR_U8_RING = 4      /* as TENSOR_U8, the node level and the children (in halves) in
                                          separate tensor-memory columns: one issuer, a three-slot ring */
};

RBW_API const char* rbw_last_error(void);
RBW_API const char* rbw_version(void);
RBW_API void rbw_build_options_default(rbw_build_options* opts);

/* Replaces rbow::impl::buildVocabularyImpl (RapidBoW.h:75-79, RapidBoW.cpp:26-41) and
 * buildSiftVocabulary (Vocabulary.cpp:32-121).  Synchronous on `stream`.  opts may be NULL
 * (reference defaults).  SIFT attributes only (uint8, L2, 128 dims); branch factor 2..16. */
RBW_API int rbw_voc_build(rbw_desc_attr attr, uint32_t branch_factor, const void* dev_desc, uint32_t nb_desc,
                          uint32_t nb_doc, uint32_t nb_levels, const rbw_build_options* opts, void* stream,
                          rbw_vocabulary** out);

/* Builds a vocabulary from host arrays: centers [levelBeg(L)][B][128] uint8, masks
 * [levelBeg(L)], weights [levelBeg(L)][B] (the fields of Vocabulary, Vocabulary.h:44-51). */
RBW_API int rbw_voc_from_host(uint32_t branch_factor, uint32_t nb_levels, const uint8_t* centers,
                              const uint32_t* masks, const float* weights, rbw_vocabulary** out);

/* rbw_voc_from_host with fp32 centers [levelBeg(L)][B][128] (no counterpart in the reference):
 * a float-center vocabulary (see RBW_BUILD_FLOAT_CENTERS). */
RBW_API int rbw_voc_from_host_f32(uint32_t branch_factor, uint32_t nb_levels, const float* centers,
                                  const uint32_t* masks, const float* weights, rbw_vocabulary** out);

/* Replaces IVocabulary::lookUp (RapidBoW.h:66-68, Vocabulary.h:59-63): leaf index per descriptor
 * in [0, B^L), asynchronous on `stream`, device buffers. */
RBW_API int rbw_voc_lookup(const rbw_vocabulary* voc, const void* dev_desc, uint32_t nb_desc, uint32_t* dev_leaf,
                           void* stream);

/* lookUp with an explicit algorithm; reports the number of kernels it launched. */
RBW_API int rbw_voc_lookup_ex(const rbw_vocabulary* voc, const void* dev_desc, uint64_t nb_desc, uint32_t* dev_leaf,
                              int32_t algo, void* stream, uint32_t* kernels_launched);

/* lookUp from host memory to host memory: copies descriptors in, looks them up and copies the
 * leaf indices back, pipelined in chunks over two streams; returns when results are on the
 * host.  Host buffers should be pinned for full PCIe bandwidth. */
RBW_API int rbw_voc_lookup_host(const rbw_vocabulary* voc, const void* host_desc, uint64_t nb_desc,
                                uint32_t* host_leaf, int32_t algo, uint32_t* kernels_launched);

/* Replaces IVocabulary::serialize (RapidBoW.h:69, Vocabulary.cpp:175-198).  With buf == NULL
 * only *size is set.  For B = 16 the bytes are the reference's blob format. */
RBW_API int rbw_voc_serialize(const rbw_vocabulary* voc, uint8_t* buf, uint64_t capacity, uint64_t* size);

/* Replaces rbow::deserializeVocabulary (RapidBoW.h:90, Vocabulary.cpp:126-157). */
RBW_API int rbw_voc_deserialize(const uint8_t* blob, uint64_t size, rbw_vocabulary** out);

/* getDescriptorAttributes / getBranchFactor / getNbLevels (RapidBoW.h:63-65). */
RBW_API int rbw_voc_info(const rbw_vocabulary* voc, rbw_desc_attr* attr, uint32_t* branch_factor, uint32_t* nb_levels,
                         uint64_t* nb_nodes);

/* Replaces IVocabularyInternal::getLevelWeights (RapidBoWInternal.h:26-31): host pointer to
 * float[levelSize(level)][B], valid for the lifetime of the vocabulary. */
RBW_API int rbw_voc_level_weights(const rbw_vocabulary* voc, uint32_t level, const float** host_weights);

/* Copies the tree out: centers [levelBeg(L)][B][128], masks [levelBeg(L)], weights
 * [levelBeg(L)][B] (any pointer may be NULL).  Test and tooling helper. */
RBW_API int rbw_voc_get_tree(const rbw_vocabulary* voc, uint8_t* host_centers, uint32_t* host_masks,
                             float* host_weights);

/* No counterpart in the reference.  *type = RBW_CENTERS_UINT8 or RBW_CENTERS_FLOAT32. */
RBW_API int rbw_voc_center_type(const rbw_vocabulary* voc, int32_t* type);

/* fp32 centers [levelBeg(L)][B][128] of a float-center vocabulary (RBW_ERR_UNSUPPORTED for a
 * uint8 one, whose centers rbw_voc_get_tree returns; for a float one that returns them rounded). */
RBW_API int rbw_voc_get_centers_f32(const rbw_vocabulary* voc, float* host_centers);

/* Statistics of the build that made the vocabulary (no counterpart in the reference). */
RBW_API int rbw_voc_build_stats(const rbw_vocabulary* voc, rbw_build_stats* stats);

/* Reads and clears how many lookup descriptors were re-scored in FP64 since the last call
 * (float-center vocabularies; 0 otherwise).  Synchronizes the device. */
RBW_API int rbw_voc_refined_lookups(const rbw_vocabulary* voc, uint64_t* refined);

/* Device scratch bytes rbw_voc_lookup needs for nb_desc descriptors. */
RBW_API int rbw_voc_lookup_scratch_bytes(const rbw_vocabulary* voc, uint64_t nb_desc, uint64_t* bytes);

/* Reads and clears the device-side error record (set by a bounded wait that timed out).
 * Synchronizes the device. */
RBW_API int rbw_voc_device_errors(const rbw_vocabulary* voc, uint32_t* code, uint32_t* where);

/* No counterpart in the reference.  rbw_voc_lookup for callers that must not allocate device
 * memory during the call (latency-bound serving loops, plug-ins inside an application that owns
 * the GPU memory, fixed memory budgets): the same tensor-core lookup, with its working memory taken from one
 * 8 MiB device array that the library reserves on each GPU for the life of the process.
 * The first call on a device resolves that array's address and must come before any stream
 * capture; the address is kept for the life of the process, so after cudaDeviceReset on that
 * device this entry point must not be used again.  Calls that may overlap on the GPU share the
 * array and race, so serialise them.
 * Calls needing more than 8 MiB of working memory (about one million descriptors for a
 * 16-ary, 4-level tree; see rbw_voc_lookup_scratch_bytes) fail with RBW_ERR_INVALID_ARG, and
 * float-center vocabularies with RBW_ERR_UNSUPPORTED. */
RBW_API int rbw_voc_lookup_noalloc(const rbw_vocabulary* voc, const void* dev_desc, uint32_t nb_desc,
                                   uint32_t* dev_leaf, void* stream);

/* Replaces IVocabulary::~IVocabulary (RapidBoW.cpp:24). */
RBW_API void rbw_voc_destroy(rbw_vocabulary* voc);

/* ------------------------------------------------------------------ inverted file
 * Replaces rbow::IDataBase (RapidBoW.h:92-107, DataBase.h:35-64, DataBase.cpp:39-197): an
 * inverted file over the leaf words of a vocabulary, scored with hierarchical tf-idf L1
 * distances.  The index lives on the GPU.  Adds are staged on the host and indexed on the
 * device at the next query, in work proportional to the documents added (a delta segment,
 * merged into the main segment from time to time), ordered with queries by CUDA events.
 * Documents, queries and max_results have no size limit beyond memory (items above 32768
 * descriptors are sorted in global memory, result sets above 1024 selected there).
 * Results are ordered by ascending score, ties by ascending document id (the reference's
 * std::sort leaves the order of equal scores unspecified). */
typedef struct rbw_database rbw_database;

/* rbow::createDataBase (RapidBoW.h:107).  The database keeps a non-owning reference to the
 * vocabulary (DataBase.h:43-45) but copies its weights, so only creation needs it. */
RBW_API int rbw_db_create(const rbw_vocabulary* voc, rbw_database** out);
RBW_API void rbw_db_destroy(rbw_database* db);

/* IDataBase::addDoc (RapidBoW.h:98, DataBase.cpp:39-69): host leaf indices of one document.
 * RBW_ERR_DUPLICATE for an index already present; RBW_ERR_INVALID_ARG for a leaf >= B^L. */
RBW_API int rbw_db_add(rbw_database* db, uint32_t idx_doc, const uint32_t* host_leaves, uint32_t n);

/* addDoc for many documents: document i owns host_leaves[offsets[i] .. offsets[i+1]).  The
 * batch is validated first; on failure nothing is added. */
RBW_API int rbw_db_add_batch(rbw_database* db, const uint32_t* doc_ids, const uint32_t* host_leaves,
                             const uint64_t* offsets, uint32_t n_docs);

/* IDataBase::query (RapidBoW.h:100-101, DataBase.cpp:71-190): host leaves in; up to
 * max_results document ids (and their scores, if out_scores is not NULL) out; *n_out results.
 * Synchronous. */
RBW_API int rbw_db_query(const rbw_database* db, const uint32_t* host_leaves, uint32_t n, uint32_t max_results,
                         uint32_t* out_docs, float* out_scores, uint32_t* n_out);

/* IDataBase::queryAndAddDoc (RapidBoW.h:103-104, DataBase.cpp:192-197). */
RBW_API int rbw_db_query_and_add(rbw_database* db, uint32_t idx_doc, const uint32_t* host_leaves, uint32_t n,
                                 uint32_t max_results, uint32_t* out_docs, float* out_scores, uint32_t* n_out);

/* Many queries in one launch (no counterpart in the reference, which scores one query per
 * call): query i owns dev_leaves[dev_offsets[i] .. dev_offsets[i+1]) (device buffers).  Writes
 * dev_docs / dev_scores [n_queries][max_results] and dev_counts [n_queries], asynchronously on
 * `stream`; the offsets are read back first (one synchronisation).  Leaves >= B^L are ignored. */
RBW_API int rbw_db_query_batched(const rbw_database* db, const uint32_t* dev_leaves, const uint64_t* dev_offsets,
                                 uint32_t n_queries, uint32_t max_results, uint32_t* dev_docs, float* dev_scores,
                                 uint32_t* dev_counts, void* stream);

/* rbw_db_query_batched with a host copy of the offsets as well, so nothing is read back and the
 * call does not wait for earlier work on `stream` (for pipelined callers). */
RBW_API int rbw_db_query_batched_host_offsets(const rbw_database* db, const uint32_t* dev_leaves,
                                              const uint64_t* dev_offsets, const uint64_t* host_offsets,
                                              uint32_t n_queries, uint32_t max_results, uint32_t* dev_docs,
                                              float* dev_scores, uint32_t* dev_counts, void* stream);

/* Number of documents and postings (descriptors) added. */
RBW_API int rbw_db_info(const rbw_database* db, uint32_t* n_docs, uint64_t* n_postings);

/* Documents in the main and delta segments of the device index, after bringing it up to date
 * (no counterpart in the reference).  Documents added since the last compaction live in the
 * delta, which is rebuilt on its own at the next query; the delta is merged into the main
 * segment once it holds more than max(256, main / 4) documents. */
RBW_API int rbw_db_segments(const rbw_database* db, uint32_t* main_docs, uint32_t* delta_docs);

/* The stored reciprocal L1 norm of a document's weight vector (DataBase.cpp:54-68). */
RBW_API int rbw_db_doc_rcp(const rbw_database* db, uint32_t idx_doc, float* rcp);

/* Subtree posting counts of every word, host [levelBeg(L)][B] (the leaf level included), as the
 * skip rule postings < 16 + 4 max_results (DataBase.cpp:125) uses them; brings the index up to
 * date first.  No counterpart in the reference. */
RBW_API int rbw_db_word_postings(const rbw_database* db, uint64_t* host_counts);
/* Makes the skip rule use host_counts (same layout) instead of this database's own counts; NULL
 * restores its own.  For a database that holds one shard of a document set: given the counts
 * summed over all shards, it skips exactly the words the whole set would, so the merged top-k of
 * the shards equals the top-k of one database holding every document.  Set it again after
 * documents are added to any shard.  No counterpart in the reference. */
RBW_API int rbw_db_set_word_postings(rbw_database* db, const uint64_t* host_counts);

/* A leaf's posting list as the reference stores it (DataBase.h:58): document ids ascending,
 * repeated once per descriptor.  *n = full length; at most `capacity` ids are written. */
RBW_API int rbw_db_postings(const rbw_database* db, uint32_t leaf, uint32_t* out, uint32_t capacity, uint32_t* n);

/* ------------------------------------------------------------------ serving
 * No counterpart in the reference, whose application looks a query image up and queries the
 * database one image at a time.  A server answers query images (host descriptors) with their
 * top-k documents (lookup + scoring) and batches them continuously: a batch is formed from the
 * waiting requests, in arrival order, as soon as one of max_inflight_batches slots is free and
 * only while its device-memory estimate fits both what the batches in flight leave of
 * hbm_budget_bytes and the device memory free at that moment (the driver's free memory plus
 * what the library's pool holds unused, less 256 MiB; this check is skipped while no batch is
 * in flight); each batch runs on its own stream, so batches overlap on the GPU and requests
 * that arrive meanwhile join the next one.  Results do not depend on the batching. */
typedef struct rbw_server rbw_server;

typedef struct {
    uint32_t max_batch_queries;     /* requests per batch (default 256) */
    uint32_t max_inflight_batches;  /* batches on the GPU at once (default 3) */
    uint64_t max_batch_descriptors; /* descriptors per batch (default 2^21) */
    uint64_t hbm_budget_bytes;      /* device memory for batches; 0 = half the free memory at creation */
    uint32_t max_results;           /* k of every request, >= 1 (default 100) */
} rbw_server_options;

typedef struct {
    uint64_t submitted, completed, batches;
    uint32_t max_inflight_seen;     /* most batches on the GPU at once */
    double mean_batch_requests;
    double p50_ms, p99_ms, max_ms;  /* latency from submit to result, completed requests */
    /* the same latency in three stages, p99 and max of each: waiting for a batch (submit to
     * dispatch), the host's launch of the batch, and the batch on the device until its result
     * is collected */
    double queue_p99_ms, launch_p99_ms, device_p99_ms;
    double queue_max_ms, launch_max_ms, device_max_ms;
} rbw_server_stats;

RBW_API void rbw_server_options_default(rbw_server_options* opts);
/* The vocabulary and database must outlive the server; documents may still be added. */
RBW_API int rbw_server_create(const rbw_vocabulary* voc, rbw_database* db, const rbw_server_options* opts,
                              rbw_server** out);
/* Copies the request's descriptors (n_desc x 128 bytes, host) and returns at once. */
RBW_API int rbw_server_submit(rbw_server* server, const void* host_desc, uint32_t n_desc, uint64_t* request_id);
/* Waits for a request (timeout_us < 0: no limit; RBW_ERR_TIMEOUT when it runs out, and the
 * request can be waited for again) and collects its results: up to `capacity` documents and
 * scores, *n_out of them in all, and its latency. */
RBW_API int rbw_server_wait(rbw_server* server, uint64_t request_id, int64_t timeout_us, uint32_t* docs,
                            float* scores, uint32_t capacity, uint32_t* n_out, double* latency_ms);
RBW_API int rbw_server_get_stats(rbw_server* server, rbw_server_stats* stats);
RBW_API int rbw_server_reset_stats(rbw_server* server);
/* The device-memory estimate the server reserves against hbm_budget_bytes for a batch of
 * n_requests requests holding n_desc descriptors in all (for sizing the budget). */
RBW_API int rbw_server_batch_bytes(rbw_server* server, uint64_t n_desc, uint32_t n_requests, uint64_t* bytes);
/* Fails requests still waiting, finishes the batches in flight. */
RBW_API void rbw_server_destroy(rbw_server* server);

/* ------------------------------------------------------------------ sharded build
 * No counterpart in the reference, which builds on one GPU (Vocabulary.cpp:32-121).  One rank's
 * part of a build whose descriptors are split across ranks (GPUs) in contiguous ranges; the
 * driver (rapidbow_b200.distributed) runs the same steps on every rank and all-reduces, between
 * rbw_kmeans_shard_assign and rbw_kmeans_shard_update, the per-node buffers of every Lloyd step:
 * sums [nodes][16][128] u64, counts [nodes][16] u32 and change counts [nodes] u32 (device
 * memory, zeroed by the caller before each assign).  The result equals the single-GPU build with
 * RBW_BUILD_IEEE_DIVISION, byte for byte. */
typedef struct rbw_kmeans_shard rbw_kmeans_shard;
RBW_API int rbw_kmeans_shard_create(const void* dev_desc, uint32_t nb_desc, uint32_t branch_factor,
                                    uint32_t nb_levels, void* stream, rbw_kmeans_shard** out);
RBW_API void rbw_kmeans_shard_destroy(rbw_kmeans_shard* shard);
/* Current level and its number of nodes (B^level). */
RBW_API int rbw_kmeans_shard_level(rbw_kmeans_shard* shard, uint32_t* level, uint32_t* nb_nodes);
/* Local members of every node of the current level (host [nb_nodes]). */
RBW_API int rbw_kmeans_shard_node_counts(rbw_kmeans_shard* shard, uint32_t* host_counts);
/* Rows of local members given as (node, position among the node's local members). */
RBW_API int rbw_kmeans_shard_member_rows(rbw_kmeans_shard* shard, const uint32_t* host_node,
                                         const uint32_t* host_pos, uint32_t count, uint8_t* host_rows);
/* Rows of local descriptors (index within this shard). */
RBW_API int rbw_kmeans_shard_desc_rows(rbw_kmeans_shard* shard, const uint32_t* host_idx, uint32_t count,
                                       uint8_t* host_rows);
/* Initial centers of the current level, host [nb_nodes][B][128]. */
RBW_API int rbw_kmeans_shard_set_centers(rbw_kmeans_shard* shard, const uint8_t* host_centers);
/* Local assign step of the nodes whose last reduced change count (dev_last_changed) is non-zero. */
RBW_API int rbw_kmeans_shard_assign(rbw_kmeans_shard* shard, const uint32_t* dev_last_changed, uint64_t* dev_sums,
                                    uint32_t* dev_counts, uint32_t* dev_changed);
/* Update from the reduced buffers (IEEE division, kmeans.cu:356-372); the buffers are only read. */
RBW_API int rbw_kmeans_shard_update(rbw_kmeans_shard* shard, const uint64_t* dev_sums, const uint32_t* dev_counts,
                                    const uint32_t* dev_changed);
RBW_API int rbw_kmeans_shard_get_centers(rbw_kmeans_shard* shard, uint8_t* host_centers);
/* Stable regroup into the next level (Vocabulary.cpp:83-98); local child counts [nb_nodes][B]. */
RBW_API int rbw_kmeans_shard_next_level(rbw_kmeans_shard* shard, uint32_t* host_child_counts);

/* The reference's initial picks (kmeans.cpp:141-196) for the nodes of one level, from node sizes:
 * positions [nb_nodes][B] among each node's members and the number of distinct picks.  One picker
 * per build: its default-seeded engine carries over from level to level, as in the reference. */
typedef struct rbw_init_picker rbw_init_picker;
RBW_API int rbw_init_picker_create(rbw_init_picker** out);
RBW_API void rbw_init_picker_destroy(rbw_init_picker* picker);
RBW_API int rbw_init_picker_level(rbw_init_picker* picker, uint32_t branch_factor, const uint32_t* node_counts,
                                  uint32_t nb_nodes, uint32_t* positions, uint32_t* n_valid);
/* Node weights from occurrence counts (Vocabulary.cpp:103-108). */
RBW_API int rbw_idf_weights(uint32_t nb_doc, const uint32_t* occ, uint64_t n, float* weights);

/* ------------------------------------------------------------------ tuning
 * No counterpart in the reference (which sizes its assign grid by an occupancy query,
 * kmeans.cu:307-322).  Launch parameters picked by an autotuner (rapidbow_b200.autotune, which
 * times the candidates on the caller's workload and keeps a per-device cache file), stored per
 * (parameter, branch factor, tree levels, descriptor-count bucket = floor(log2(n))); levels 0
 * matches any depth.  Unset entries use the defaults. */
enum {
    RBW_TUNE_ASSIGN_CTAS_PER_SM = 0,     /* uint8 k-means assign: CTAs per SM, 1..8 (default 6) */
    RBW_TUNE_ASSIGN_F32_CTAS_PER_SM = 1, /* float-center assign: CTAs per SM, 1..3 (default 3) */
    RBW_TUNE_SCATTER_ROWS = 2,           /* lookup regroup: rows per thread, 8, 16 or 32 (default 16) */
    RBW_TUNE_DB_SHARD_TABLES = 3,        /* DataBase inverted file, keyed by documents instead of
                                            descriptors: 1 grouped tables per 2,560-document shard
                                            while those tables stay small (default), 2 one CSR */
    RBW_TUNE_LOOKUP_SCHEDULE = 4,        /* the tensor-core schedule RBW_LOOKUP_AUTO runs: 1 level
                                            pairs in two buffers (default), 2 the three-slot ring */
    RBW_TUNE_ASSIGN_SUMS = 5             /* uint8 k-means center sums: 1 shared-memory atomics
                                            (default), 2 a second MMA per tile (at most 4 CTAs/SM) */
};
/* value 0 removes the entry; RBW_ERR_INVALID_ARG for a value the parameter cannot take. */
RBW_API int rbw_tuning_set(uint32_t param, uint32_t branch_factor, uint32_t nb_levels, uint32_t bucket,
                           uint32_t value);
/* The value a launch for n descriptors would use. */
RBW_API int rbw_tuning_get(uint32_t param, uint32_t branch_factor, uint32_t nb_levels, uint64_t n, uint32_t* value);
RBW_API int rbw_tuning_clear(void);

/* Optional CUDA-event timing of this library's own kernel launches (no reference
 * counterpart; used by bench.py).  While enabled, each launch of a timed kernel is bracketed by
 * two events on its stream.  rbw_timing_read sums completed launches of one kernel id:
 * 0 lookup tensor pass, 1 lookup FP32 SIMT, 2 lookup regroup, 3 k-means assign,
 * 4 k-means update, 5 scoring (all of it), 6 inverted-file construction, 7 query preparation
 * and 8 candidate merge (both also inside 5).  Read after synchronising. */
RBW_API void rbw_timing_enable(int32_t on);
RBW_API int rbw_timing_reset(void);
RBW_API int rbw_timing_read(uint32_t kernel, double* total_ms, uint64_t* launches);

#ifdef __cplusplus
}
#endif
#endif
