/* Test infrastructure only: the oracle (CPU restatement of the reference algorithm).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may load this library,
 * and only as the checker / the timed CPU baseline -- never as the product path.
 *
 * Layouts (shared with the product):
 *   descriptors : uint8 [n][128], row-major.
 *   centers     : uint8 [levelBeg(L)][B][128]; node index = breadth-first (levelBeg(l) + i).
 *                 For B = 16 this is the reference's Node (uint32[32 words][16 centers],
 *                 Vocabulary.h:42) with word w of center j = bytes 4w..4w+3 of row j.
 *   masks       : uint32 [levelBeg(L)], bit b = center b was a distinct initial pick.
 *   weights     : float  [levelBeg(L)][B] (Vocabulary.h:86 for B = 16).
 *   leaf index  : uint32 in [0, B^L) (Vocabulary.h:59-63).
 */
#ifndef RBW_ORACLE_H
#define RBW_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

uint64_t orc_level_beg(uint32_t B, uint32_t level);

/* Tree descent (vocTreeLookUp.cu:82-155): exact integer squared L2, lowest branch on ties. */
void orc_lookup(const uint8_t* centers, uint32_t B, uint32_t L, const uint8_t* desc, uint64_t n,
                uint32_t* out, uint32_t nThreads);

/* One k-means assign over one node (kmeans.cu:95-199, tests/KmeansAssignCenterTests.cpp:147-189).
 * members: descriptor indices (n of them); assign: in = previous, out = new; counts[B],
 * sums[B][128] (uint64, accumulated), nbChanged accumulated. */
void orc_kmeans_assign(const uint8_t* desc, const uint32_t* members, uint32_t n, const uint8_t* centers,
                       uint32_t B, uint8_t* assign, uint32_t* counts, uint64_t* sums, uint32_t* nbChanged);

/* Center update (kmeans.cu:356-372): c = (uint8) roundf(float(sum) / float(count)) for count > 0.
 * The reference divides with the fast approximate division (--use_fast_math); the oracle divides
 * with IEEE division, which can differ only when sum/count is within a few ulp of k + 0.5. */
void orc_kmeans_update(const uint32_t* counts, const uint64_t* sums, uint32_t B, uint8_t* centers);

enum { ORC_INIT_REFERENCE = 0, ORC_INIT_KMEANSPP = 1, ORC_INIT_INJECTED = 2 };

/* Initial centers of one node for ORC_INIT_KMEANSPP: seeded k-means++ over <= 256 sampled members.
 * SplitMix64 stream seeded with seed ^ level * 0x9E3779B97F4A7C15 ^ node * 0xD1B54A32D192ED03; Floyd
 * sampling of min(n, 256) member positions (sorted); the first center uniform over the sample;
 * then D^2 sampling with exact integer squared distances (smallest i with prefix > draw % total);
 * stops early when every sampled member coincides with a chosen center.  Padding repeats the last
 * pick.  Returns the number of distinct picks. */
uint32_t orc_kmeanspp_init(const uint8_t* desc, const uint32_t* members, uint32_t n, uint32_t B,
                           uint64_t seed, uint32_t level, uint64_t nodeInLevel, uint32_t* pickedDesc);

/* Hierarchical k-means vocabulary build (Vocabulary.cpp:32-121, kmeans.cpp:27-225).
 *   maxIter : Lloyd cap (reference default 1000);
 *   initMode: ORC_INIT_REFERENCE (randPick with a fresh default-seeded mt19937_64,
 *             kmeans.cpp:141-196), ORC_INIT_KMEANSPP (seeded), ORC_INIT_INJECTED (injected[],
 *             B descriptor indices per node in breadth-first order; UINT32_MAX = invalid).
 *   outputs : centers, masks, weights as documented above; occ [levelBeg(L)][B];
 *             itersOut [levelBeg(L)] = Lloyd iterations each node ran (may be NULL).
 * Returns 0, or -1 when nbDesc < B or nbDoc == 0 (Vocabulary.cpp:39-44). */
int orc_build_vocabulary(const uint8_t* desc, uint32_t nbDesc, uint32_t nbDoc, uint32_t B, uint32_t L,
                         uint32_t maxIter, uint32_t initMode, uint64_t seed, const uint32_t* injected,
                         uint8_t* centers, uint32_t* masks, float* weights, uint32_t* occ, uint32_t* itersOut);

/* ---- Float-center mode (no counterpart in the reference, whose centers are uint8: kmeans.cu:367).
 * It generalises the reference's assign/update (kmeans.cu:125-199, 356-372) to fp32 centers:
 *   distance : FP64 squared L2 in one fixed evaluation order, identical on the GPU (orc_dist64);
 *   assign   : argmin of that distance, lowest index on ties (kmeans.cu:131-135);
 *   update   : c = float(double(sum) / double(count)) from exact integer sums, kept when count = 0;
 *   inertia  : FP64 sum over the members of their distance to the assigned center.
 * Initial centers are the same descriptor rows as in the uint8 mode (converted exactly).
 * Parity unpinned: the reference has no float-center mode to run or to take vectors from; this
 * part is checked against itself (plain FP64 sums, integer trees equal to the uint8 restatement,
 * independence from the thread count) and shares the uint8 mode's pinned rules. */

/* Squared distance of a uint8 row to an fp32 center: lane l (0..31) forms
 * p_l = fma(e, e, .) over e = double(x[4l+k]) - double(c[4l+k]), k = 0..3 (starting from 0);
 * then for off = 16, 8, 4, 2, 1: p_l = p_l + p_(l xor off); the result is p_0. */
double orc_dist64(const uint8_t* x, const float* c);

/* Tree descent through fp32 centers [levelBeg(L)][B][128] with orc_dist64. */
void orc_lookup_f32(const float* centers, uint32_t B, uint32_t L, const uint8_t* desc, uint64_t n,
                    uint32_t* out, uint32_t nThreads);

/* Float-center hierarchical build, same level loop, init modes and freezing rule as
 * orc_build_vocabulary.  centers: float [levelBeg(L)][B][128].  inertiaFirst / inertiaLast
 * [L]: the level's inertia (sum over its nodes) after its first and after its last Lloyd step
 * (frozen nodes keep their last value); either may be NULL. */
int orc_build_vocabulary_f32(const uint8_t* desc, uint32_t nbDesc, uint32_t nbDoc, uint32_t B, uint32_t L,
                             uint32_t maxIter, uint32_t initMode, uint64_t seed, const uint32_t* injected,
                             float* centers, uint32_t* masks, float* weights, uint32_t* occ, uint32_t* itersOut,
                             double* inertiaFirst, double* inertiaLast, uint32_t nThreads);

/* Inverted file + scoring (DataBase.cpp:39-197), B = branching, L = levels. */
void* orc_db_create(uint32_t B, uint32_t L, const float* weights);
void orc_db_destroy(void* db);
/* Returns 0, or -1 on a duplicate document index (DataBase.cpp:41-43). */
int orc_db_add(void* db, uint32_t idxDoc, const uint32_t* leaves, uint32_t n);
/* Reciprocal L1 norm stored for a document (DataBase.cpp:54-68): float(1 / sum in double). */
float orc_db_doc_rcp(const void* db, uint32_t idxDoc);
/* Query (DataBase.cpp:71-190).  mode 0 = reference arithmetic (float terms, double
 * accumulator, float score); mode 1 = FP64 throughout.  Writes every touched document:
 * docs/scores sorted by (score ascending, doc ascending); returns the count (<= capacity). */
uint32_t orc_db_query(const void* db, const uint32_t* leaves, uint32_t n, uint32_t maxNbResults,
                      int mode, uint32_t* docs, double* scores, uint32_t capacity);
/* Subtree posting counts of every word ([levelBeg(L)][B]), and counts the skip rule uses instead
 * of the database's own (NULL: its own) -- for a database holding one shard of a document set. */
void orc_db_word_postings(const void* db, uint64_t* out);
void orc_db_set_word_postings(void* db, const uint64_t* counts);
/* Postings of one leaf word, sorted ascending with duplicates (= term frequency). */
uint32_t orc_db_postings(const void* db, uint32_t leaf, uint32_t* out, uint32_t capacity);

#ifdef __cplusplus
}
#endif
#endif
