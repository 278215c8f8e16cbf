/*
 * wc_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of warpcore's hot path
 * (include/warpcore/{hashers,probing_schemes,base,status,
 * single_value_hash_table,hash_set,counting_hash_table,bloom_filter}.cuh)
 * used as the checker for the CUDA library in warpcore_b200/.  It reproduces
 * the reference's exact probe order (unaligned cooperative-group windows,
 * lane order of CAS attempts), so it also gives the reference's slot
 * placement for a given insertion order.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may
 * load this code.  The product path never calls it.
 *
 * Parity pin: the hashers, the capacity rule and the prime table are checked
 * against golden fixtures produced from the reference's own sources
 * (tests/golden/), and the table/filter results against fixtures produced by
 * the reference's CUDA code run on a B200 (tests/golden/make_golden.cu).
 */
#ifndef WC_ORACLE_H
#define WC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* hasher ids (hashers.cuh:14-175) */
enum {
    WCO_HASH_MURMUR = 0,     /* MurmurHash<K>: fmix32 / fmix64, hash type = K */
    WCO_HASH_NVIDIA = 1,     /* NvidiaHash, u32 only */
    WCO_HASH_MUELLER = 2,    /* MuellerHash, u32 only */
    WCO_HASH_IDENTITY32 = 3, /* IdentityMap<K, uint32_t> */
    WCO_HASH_IDENTITY64 = 4  /* IdentityMap<K, uint64_t> */
};

/* probing scheme ids (probing_schemes.cuh:22-305) */
enum {
    WCO_PROBE_DOUBLE = 0,
    WCO_PROBE_LINEAR = 1,
    WCO_PROBE_QUADRATIC = 2
};

/* table kinds */
enum {
    WCO_SVHT = 0,
    WCO_HASHSET = 1,
    WCO_COUNTING = 2,
    WCO_MULTIVALUE = 3
};

/* Status bits (status.cuh:44-68) */
#define WCO_ST_NONE                    0u
#define WCO_ST_UNKNOWN_ERROR           (1u << 0)
#define WCO_ST_PROBING_LENGTH_EXCEEDED (1u << 1)
#define WCO_ST_INVALID_CONFIGURATION   (1u << 2)
#define WCO_ST_INVALID_KEY             (1u << 3)
#define WCO_ST_DUPLICATE_KEY           (1u << 4)
#define WCO_ST_KEY_NOT_FOUND           (1u << 5)
#define WCO_ST_INDEX_OVERFLOW          (1u << 6)
#define WCO_ST_OUT_OF_MEMORY           (1u << 7)
#define WCO_ST_NOT_INITIALIZED         (1u << 8)
#define WCO_ST_DRY_RUN                 (1u << 9)
#define WCO_ST_INVALID_PHASE_OVERLAP   (1u << 10)
#define WCO_ST_MAX_VALUES_REACHED      (1u << 11)
#define WCO_ST_INVALID_VALUE           (1u << 12)

/* ---- hashers ---- */
uint64_t wco_hash(int hasher, int key_bytes, uint64_t x);
int wco_hash_bits(int hasher, int key_bytes);

/* ---- prime table and capacity rule (base.cuh:27-34, primes.hpp) ---- */
uint64_t wco_num_primes(void);
void wco_primes(uint64_t *out);
uint64_t wco_valid_capacity(uint64_t min_capacity, uint64_t cg_size);

/* ---- probe sequence of one key, reference order ----
 * out[w * cg + r] = slot probed by lane r in window w; returns #windows */
uint64_t wco_probe_sequence(int scheme, int h1, int h2, int key_bytes,
                            uint64_t cg, uint64_t capacity, uint64_t key,
                            uint64_t seed, uint64_t probing_length,
                            uint64_t max_windows, uint64_t *out);

/* ---- status handler ReturnBoolean<Ignore> (status.cuh:316-330) ---- */
uint8_t wco_status_to_bool(uint32_t status, uint32_t ignore);

/* ---- open-addressing tables ---- */
typedef struct wco_table wco_table;

wco_table *wco_table_create(int kind, int key_bytes, int value_bytes,
                            uint64_t min_capacity, uint64_t seed, uint64_t cg,
                            int scheme, int h1, int h2, uint64_t empty_key,
                            uint64_t tombstone_key, uint64_t max_count);
void wco_table_destroy(wco_table *t);
uint64_t wco_table_capacity(const wco_table *t);
void wco_table_init(wco_table *t, uint64_t seed);

/* status_out may be NULL; otherwise one uint32 Status per key */
void wco_insert(wco_table *t, const void *keys, const void *values, uint64_t n,
                uint64_t probing_length, uint32_t *status_out);
/* SVHT / counting: values_out written only on a hit (gpu_engine.cuh:252-257);
 * hash set: values_out is uint8 flags, written when the status is none */
void wco_retrieve(wco_table *t, const void *keys, uint64_t n, void *values_out,
                  uint64_t probing_length, uint32_t *status_out);
void wco_erase(wco_table *t, const void *keys, uint64_t n,
               uint64_t probing_length, uint32_t *status_out);
uint64_t wco_size(const wco_table *t);
uint64_t wco_retrieve_all(const wco_table *t, void *keys_out, void *values_out);
uint32_t wco_peek_status(const wco_table *t);
uint32_t wco_pop_status(wco_table *t);
/* raw slot arrays (keys and values widened to uint64) */
void wco_table_slots(const wco_table *t, uint64_t *keys_out, uint64_t *values_out);

/* ---- pattern-blocked Bloom filter (bloom_filter.cuh) ---- */
/* MultiValueHashTable (multi_value_hash_table.cuh) */
wco_table *wco_mv_create(int key_bytes, int value_bytes, uint64_t min_capacity, uint64_t seed,
                         uint64_t cg, int scheme, int h1, int h2, uint64_t empty_key,
                         uint64_t tombstone_key, uint64_t max_values_per_key);
void wco_mv_insert(wco_table *t, const void *keys, const void *values, uint64_t n,
                   uint64_t probing_length, uint32_t *status_out);
uint64_t wco_mv_num_values(wco_table *t, const void *keys, uint64_t n, uint64_t *counts_out,
                           uint64_t probing_length, uint32_t *status_out);
uint64_t wco_mv_retrieve(wco_table *t, const void *keys, uint64_t n, uint64_t *begin_out,
                         uint64_t *end_out, void *values_out, uint64_t probing_length,
                         uint32_t *status_out);
uint64_t wco_mv_num_keys(const wco_table *t);
uint64_t wco_mv_unique_keys(const wco_table *t, void *keys_out);

/* BucketListHashTable (bucket_list_hash_table.cuh) with
 * BucketListStore<Value, index_bits, counter_bits, size_bits>; CG cg,
 * MurmurHash double hashing, default sentinels */
typedef struct wco_bl wco_bl;
wco_bl *wco_bl_create(int key_bytes, int value_bytes, uint64_t key_capacity,
                      uint64_t value_capacity, uint64_t seed, float grow_factor,
                      uint64_t min_bucket_size, uint64_t max_bucket_size,
                      uint64_t max_values_per_key, uint64_t index_bits, uint64_t counter_bits,
                      uint64_t size_bits, uint64_t cg);
void wco_bl_destroy(wco_bl *b);
void wco_bl_init(wco_bl *b, uint64_t seed);
uint64_t wco_bl_key_capacity(const wco_bl *b);
void wco_bl_insert(wco_bl *b, const void *keys, const void *values, uint64_t n,
                   uint64_t probing_length, uint32_t *status_out);
uint64_t wco_bl_num_values(wco_bl *b, const void *keys, uint64_t n, uint64_t *counts_out,
                           uint64_t probing_length, uint32_t *status_out);
uint64_t wco_bl_retrieve(wco_bl *b, const void *keys, uint64_t n, uint64_t *begin_out,
                         uint64_t *end_out, void *values_out, uint64_t probing_length,
                         uint32_t *status_out);
uint64_t wco_bl_num_keys(const wco_bl *b);
uint64_t wco_bl_total_values(const wco_bl *b);
uint64_t wco_bl_next_free(const wco_bl *b);
uint64_t wco_bl_all_keys(const wco_bl *b, void *keys_out);
uint32_t wco_bl_peek_status(const wco_bl *b);
uint32_t wco_bl_pop_status(wco_bl *b);

/* MultiBucketHashTable (multi_bucket_hash_table.cuh); bucket <= cg */
typedef struct wco_mb wco_mb;
wco_mb *wco_mb_create(int key_bytes, int value_bytes, uint64_t bucket, uint64_t min_capacity,
                      uint64_t seed, uint64_t cg, int scheme, int h1, int h2, uint64_t empty_key,
                      uint64_t tombstone_key, uint64_t empty_value, uint64_t max_values_per_key);
void wco_mb_destroy(wco_mb *t);
uint64_t wco_mb_capacity(const wco_mb *t);
void wco_mb_init(wco_mb *t, uint64_t seed);
void wco_mb_insert(wco_mb *t, const void *keys, const void *values, uint64_t n,
                   uint64_t probing_length, uint32_t *status_out);
uint64_t wco_mb_num_values(wco_mb *t, const void *keys, uint64_t n, uint64_t *counts_out,
                           uint64_t probing_length, uint32_t *status_out);
uint64_t wco_mb_retrieve(wco_mb *t, const void *keys, uint64_t n, uint64_t *begin_out,
                         uint64_t *end_out, void *values_out, uint64_t probing_length,
                         uint32_t *status_out);
uint64_t wco_mb_num_keys(const wco_mb *t);
uint64_t wco_mb_num_occupied(const wco_mb *t);
uint64_t wco_mb_size(const wco_mb *t);
uint64_t wco_mb_unique_keys(const wco_mb *t, void *keys_out);
uint32_t wco_mb_peek_status(const wco_mb *t);
uint32_t wco_mb_pop_status(wco_mb *t);

/* Zipf draws, one splitmix64 stream per output (the library's generator) */
void wco_gen_zipf_streams(const void *in, uint64_t n_in, void *out, uint64_t n_out, int bytes,
                          double s, uint64_t seed);

typedef struct wco_bloom wco_bloom;
wco_bloom *wco_bloom_create(int key_bytes, int slot_bytes, uint64_t cg,
                            int hasher, uint64_t num_bits, uint64_t k,
                            uint64_t seed);
void wco_bloom_destroy(wco_bloom *b);
void wco_bloom_insert(wco_bloom *b, const void *keys, uint64_t n);
void wco_bloom_retrieve(const wco_bloom *b, const void *keys, uint64_t n,
                        uint8_t *flags_out);
uint64_t wco_bloom_num_slots(const wco_bloom *b);
uint64_t wco_bloom_num_blocks(const wco_bloom *b);
/* words widened to uint64 */
void wco_bloom_words(const wco_bloom *b, uint64_t *out);
double wco_bloom_fpr(const wco_bloom *b, uint64_t n);

/* ---- seeded synthetic data (splitmix64 based) ---- */
uint64_t wco_splitmix64(uint64_t *state);
/* n distinct keys, none equal to 0 or all-ones in key width */
void wco_gen_unique_keys(int key_bytes, uint64_t n, uint64_t seed, void *out);
void wco_gen_uniform(int bytes, uint64_t n, uint64_t seed, void *out);
/* Zipf(s) rejection sampler over ranks 1..n_in (random_distributions.cuh:
 * 285-310, with rank index k-1 so that it never reads past the input) */
void wco_gen_zipf_ranks(uint64_t n_in, double s, uint64_t n_out, uint64_t seed,
                        uint64_t *ranks_out);

/* ---- multi-threaded CPU port (the timed CPU baseline) ----
 * Same hasher, DoubleHashing windows and lane order as the reference, with
 * atomic CAS on the key word from `threads` pthreads.  Returns seconds. */
typedef struct wco_mt_table wco_mt_table;
wco_mt_table *wco_mt_create(int key_bytes, int value_bytes, uint64_t capacity,
                            uint64_t cg, uint64_t seed);
void wco_mt_destroy(wco_mt_table *t);
void wco_mt_clear(wco_mt_table *t, int threads);
double wco_mt_insert(wco_mt_table *t, const void *keys, const void *values,
                     uint64_t n, int threads);
double wco_mt_retrieve(wco_mt_table *t, const void *keys, uint64_t n,
                       void *values_out, uint8_t *found_out, int threads);

#ifdef __cplusplus
}
#endif

#endif /* WC_ORACLE_H */
