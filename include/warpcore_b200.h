/*
 * warpcore_b200.h -- C ABI of the B200-native warpcore library.
 *
 * The reference (sleeepyjack/warpcore) is a header-only C++ template library
 * with no C ABI; its host "bulk" methods are the boundary this library
 * replaces.  Each entry point below names the reference method it stands in
 * for (paths relative to the warpcore project).  The C++ drop-in headers in
 * include/warpcore/ call these functions; foreign callers (ctypes, cgo, JNI)
 * bind them directly.
 *
 * Conventions
 *  - Every function returns an int error code (WC_OK == 0) and never throws.
 *    A short message for the last failure on the calling thread is in
 *    wc_last_error().
 *  - Key, value, status and flag buffers are DEVICE pointers owned by the
 *    caller, exactly like the reference's bulk methods.
 *  - Bulk operations are asynchronous on the given stream (NULL = legacy
 *    default stream).  size, retrieve_all, peek_status, pop_status,
 *    *_create and *_init synchronise that stream, as the reference does.
 *  - probing_length is the reference's maximum number of probed slots per
 *    key; the library probes at most ceil(probing_length / cg_size) windows
 *    and never more windows than the table has, so a full table reports
 *    WC_STATUS_PROBING_LENGTH_EXCEEDED instead of spinning.
 *  - Per-key status output (status_out, may be NULL) follows the reference's
 *    status handlers: WC_HANDLER_NOTHING (ReturnNothing), WC_HANDLER_STATUS
 *    (ReturnStatus: one uint32 Status per key) and WC_HANDLER_BOOLEAN
 *    (ReturnBoolean<ignore>: one byte per key, computed with the reference's
 *    own Status algebra, status.cuh:142-146 and :316-330).
 */
#ifndef WARPCORE_B200_H
#define WARPCORE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t without pulling in the CUDA headers */
typedef struct CUstream_st *wc_stream_t;

/* ---- error codes ---- */
#define WC_OK 0
#define WC_ERR_INVALID_ARGUMENT (-1)
#define WC_ERR_CUDA (-2)
#define WC_ERR_OUT_OF_MEMORY (-3)
#define WC_ERR_NOT_INITIALIZED (-4)
#define WC_ERR_UNSUPPORTED (-5)
#define WC_ERR_TIMEOUT (-6) /* a bounded device-side wait ran out */

/* ---- Status bits: identical to warpcore::Status (status.cuh:44-68) ---- */
#define WC_STATUS_NONE 0u
#define WC_STATUS_UNKNOWN_ERROR (1u << 0)
#define WC_STATUS_PROBING_LENGTH_EXCEEDED (1u << 1)
#define WC_STATUS_INVALID_CONFIGURATION (1u << 2)
#define WC_STATUS_INVALID_KEY (1u << 3)
#define WC_STATUS_DUPLICATE_KEY (1u << 4)
#define WC_STATUS_KEY_NOT_FOUND (1u << 5)
#define WC_STATUS_INDEX_OVERFLOW (1u << 6)
#define WC_STATUS_OUT_OF_MEMORY (1u << 7)
#define WC_STATUS_NOT_INITIALIZED (1u << 8)
#define WC_STATUS_DRY_RUN (1u << 9)
#define WC_STATUS_INVALID_PHASE_OVERLAP (1u << 10)
#define WC_STATUS_MAX_VALUES_FOR_KEY_REACHED (1u << 11)
#define WC_STATUS_INVALID_VALUE (1u << 12)

/* ---- per-key status handlers (status.cuh:278-333) ---- */
#define WC_HANDLER_NOTHING 0
#define WC_HANDLER_STATUS 1
#define WC_HANDLER_BOOLEAN 2

/* ---- hashers (hashers.cuh:14-175) ---- */
#define WC_HASH_MURMUR 0     /* MurmurHash<Key> */
#define WC_HASH_NVIDIA 1     /* NvidiaHash (32-bit keys) */
#define WC_HASH_MUELLER 2    /* MuellerHash (32-bit keys) */
#define WC_HASH_IDENTITY32 3 /* IdentityMap<Key, uint32_t> */
#define WC_HASH_IDENTITY64 4 /* IdentityMap<Key, uint64_t> */

/* ---- probing schemes (probing_schemes.cuh:22-305) ---- */
#define WC_PROBING_DOUBLE 0    /* DoubleHashing<H1, H2, CG> */
#define WC_PROBING_LINEAR 1    /* LinearProbing<H, CG> */
#define WC_PROBING_QUADRATIC 2 /* QuadraticProbing<H, CG> */

/* Template knobs of SingleValueHashTable / HashSet / CountingHashTable
 * (single_value_hash_table.cuh:29-37, hash_set.cuh:16-22,
 * counting_hash_table.cuh:18-26) as run-time values. */
typedef struct wc_table_config {
    uint32_t key_bytes;     /* 4 or 8 */
    uint32_t value_bytes;   /* 4 or 8, with either key width; 0 for a hash set */
    uint64_t empty_key;     /* EmptyKey, default 0 */
    uint64_t tombstone_key; /* TombstoneKey, default ~0 */
    uint32_t probing;       /* WC_PROBING_* */
    uint32_t hasher1;       /* WC_HASH_*, probing hash */
    uint32_t hasher2;       /* WC_HASH_*, step hash (double hashing) */
    uint32_t cg_size;       /* cooperative group size = probe window width
                               in slots: 1, 2, 4, 8, 16 or 32 */
} wc_table_config;

/* Read-only description of a table, for the device-side per-key API. */
typedef struct wc_table_info {
    uint32_t kind;          /* 0 single-value, 1 hash set, 2 counting */
    uint32_t key_bytes, value_bytes, slot_bytes, cg_size;
    uint32_t probing, hasher1, hasher2;
    uint64_t capacity;      /* slots, reference capacity rule */
    uint64_t num_buckets;   /* capacity / cg_size */
    uint64_t seed, empty_key, tombstone_key, max_count;
    uint64_t bytes_total;
    void *slots;            /* device pointer to the slot array */
    uint32_t *status;       /* device pointer to the table's Status word */
    int is_initialized;
    unsigned char *fingerprints; /* device pointer to one byte per slot, or NULL:
                                    0 empty, 1 tombstone, else the key's
                                    fingerprint; writers of slot keys keep it */
    unsigned long long *num_keys; /* multi-value tables: device counter of keys
                                     holding a value (NULL for other kinds) */
    uint64_t max_values_per_key;  /* multi-value tables */
    unsigned long long *live;     /* device: the valid-key counters, 32 of them
                                     32 bytes apart (NULL for multi-value
                                     tables); writers of slot keys keep them */
    void *values;                 /* struct-of-arrays single-value tables: the
                                     value array, one value per key slot of
                                     `slots`; NULL for every other table */
} wc_table_info;

typedef struct wc_table wc_table;

/* last error message of the calling thread ("" if none) */
const char *wc_last_error(void);
/* kernels this library has launched in this process, over all devices and
 * streams (a batch's CUDA graph counts its one kernel) */
int wc_launch_count(uint64_t *out);
/* library version string */
const char *wc_version(void);

/* Default knobs of each table kind: MurmurHash, DoubleHashing, sentinels
 * 0 / ~0 and CG 8 (single-value), 16 (hash set), 4 (counting)
 * (defaults.cuh:11-42). */
void wc_svht_default_config(wc_table_config *cfg, uint32_t key_bytes,
                            uint32_t value_bytes);
void wc_hashset_default_config(wc_table_config *cfg, uint32_t key_bytes);
void wc_counting_default_config(wc_table_config *cfg, uint32_t key_bytes,
                                uint32_t value_bytes);

/* Capacity rule of the reference: detail::get_valid_capacity
 * (base.cuh:27-34 with primes.hpp). 0 if min_capacity is beyond the table. */
uint64_t wc_valid_capacity(uint64_t min_capacity, uint64_t cg_size);

/* ------------------------------------------------------------------ */
/* SingleValueHashTable<Key, Value, ...>                               */
/* ------------------------------------------------------------------ */

/* SingleValueHashTable(min_capacity, seed, no_init)
 * (single_value_hash_table.cuh:112-128) */
int wc_svht_create(const wc_table_config *cfg, uint64_t min_capacity,
                   uint64_t seed, int no_init, wc_table **out);
/* SingleValueHashTable<Key, Value, ..., storage::key_value::SoAStore<Key,
 * Value>> (storage.cuh:218-432): the same table stored as a struct of
 * arrays.  The slot array (wc_table_info.slots) holds the keys only,
 * capacity of them; the values sit in a separate array
 * (wc_table_info.values), value i belonging to key slot i.  An insert
 * claims the key slot with a compare-and-swap and then writes the value, as
 * the reference's SoA store does; every operation, status and answer is the
 * same as the AoS table's.  These tables keep no fingerprints, run the
 * window kernel only, and are not accepted by the batch, served and
 * persistent-server calls (WC_ERR_UNSUPPORTED / WC_ERR_INVALID_ARGUMENT). */
int wc_svht_create_soa(const wc_table_config *cfg, uint64_t min_capacity,
                       uint64_t seed, int no_init, wc_table **out);
/* ~SingleValueHashTable (single_value_hash_table.cuh:162-169); also destroys
 * hash sets and counting tables */
int wc_table_destroy(wc_table *t);
/* init(seed, stream) (single_value_hash_table.cuh:176-192); hash sets and
 * counting tables too (hash_set.cuh:161-175, counting_hash_table.cuh:114-124) */
int wc_table_init(wc_table *t, uint64_t seed, wc_stream_t stream);
/* insert(keys_in, values_in, num_in, stream, probing_length, status_out)
 * (single_value_hash_table.cuh:241-258) */
int wc_svht_insert(wc_table *t, const void *keys_in, const void *values_in,
                   uint64_t num_in, wc_stream_t stream,
                   uint64_t probing_length, void *status_out,
                   int status_handler, uint32_t ignore);
/* retrieve(keys_in, num_in, values_out, stream, probing_length, status_out)
 * (single_value_hash_table.cuh:320-337); values_out is written on hits only */
int wc_svht_retrieve(wc_table *t, const void *keys_in, uint64_t num_in,
                     void *values_out, wc_stream_t stream,
                     uint64_t probing_length, void *status_out,
                     int status_handler, uint32_t ignore);
/* erase(keys_in, num_in, stream, probing_length, status_out)
 * (single_value_hash_table.cuh:480-496) */
int wc_svht_erase(wc_table *t, const void *keys_in, uint64_t num_in,
                  wc_stream_t stream, uint64_t probing_length,
                  void *status_out, int status_handler, uint32_t ignore);
/* No counterpart in the reference, whose tables always allocate their own
 * memory (storage.cuh:464-516).  Device bytes a single-value table of this
 * configuration takes when placed on caller memory: its slots, the Status
 * word and counters, and its fingerprints if the fingerprint policy gives
 * them to it. */
int wc_svht_memory_bytes(const wc_table_config *cfg, uint64_t min_capacity, uint64_t *bytes_out);
/* A single-value table placed on caller-provided device memory (256-byte
 * aligned, at least wc_svht_memory_bytes); wc_table_destroy does not free
 * it.  no_init 0: initialise (as wc_svht_create); 1: leave uninitialised;
 * 2: adopt the memory's contents, a copy of the memory of a table of the
 * same configuration (a table swapped out to the host and back).  Works on
 * `stream` and synchronises it.  This is how a serving loop keeps tables in
 * a memory pool of its own and moves them in and out of a device budget. */
int wc_svht_create_on(const wc_table_config *cfg, uint64_t min_capacity, uint64_t seed,
                      int no_init, void *memory, uint64_t memory_bytes, wc_stream_t stream,
                      wc_table **out);
/* size(stream) (single_value_hash_table.cuh:535-592); blocking.  The
 * reference counts the valid keys with a scan of the whole slot array; here
 * single-value, set and counting tables keep a count that every claim of an
 * empty slot and every erase maintains (bulk kernels, batches and the device
 * per-key API alike), and size reads 256 bytes of counters.  Multi-value
 * tables (kind 3) count by scan. */
int wc_table_size(wc_table *t, wc_stream_t stream, uint64_t *size_out);
/* the same count by a scan of the slot array (the reference's method, kept
 * to check the maintained count); blocking */
int wc_table_size_scan(wc_table *t, wc_stream_t stream, uint64_t *size_out);
/* retrieve_all(keys_out, values_out, num_out, stream)
 * (single_value_hash_table.cuh:391-417, hash_set.cuh:367-384); blocking;
 * values_out may be NULL and is ignored for hash sets.  The outputs must
 * hold size() entries; the order of the pairs is unspecified, as in the
 * reference. */
int wc_table_retrieve_all(wc_table *t, void *keys_out, void *values_out,
                          uint64_t *num_out, wc_stream_t stream);
/* peek_status(stream) / pop_status(stream)
 * (single_value_hash_table.cuh:646-687); blocking */
int wc_table_peek_status(wc_table *t, wc_stream_t stream, uint32_t *out);
int wc_table_pop_status(wc_table *t, wc_stream_t stream, uint32_t *out);
/* capacity(), bytes_total(), seed(), is_initialized() and the device view */
int wc_table_get_info(const wc_table *t, wc_table_info *info);

/* ------------------------------------------------------------------ */
/* HashSet<Key, ...>                                                   */
/* ------------------------------------------------------------------ */

/* HashSet(min_capacity, seed) (hash_set.cuh:81-110) */
int wc_hashset_create(const wc_table_config *cfg, uint64_t min_capacity,
                      uint64_t seed, wc_table **out);
/* insert(keys_in, num_in, stream, probing_length, status_out)
 * (hash_set.cuh:266-282) */
int wc_hashset_insert(wc_table *t, const void *keys_in, uint64_t num_in,
                      wc_stream_t stream, uint64_t probing_length,
                      void *status_out, int status_handler, uint32_t ignore);
/* retrieve(keys_in, num_in, flags_out, stream, probing_length, status_out)
 * (hash_set.cuh:342-359 host form; the device form :292-329 it launches);
 * flags_out is one byte per key (C++ bool), written when the key's status
 * is none */
int wc_hashset_retrieve(wc_table *t, const void *keys_in, uint64_t num_in,
                        uint8_t *flags_out, wc_stream_t stream,
                        uint64_t probing_length, void *status_out,
                        int status_handler, uint32_t ignore);
/* erase(keys_in, num_in, stream, probing_length, status_out)
 * (hash_set.cuh:450-462) */
int wc_hashset_erase(wc_table *t, const void *keys_in, uint64_t num_in,
                     wc_stream_t stream, uint64_t probing_length,
                     void *status_out, int status_handler, uint32_t ignore);

/* ------------------------------------------------------------------ */
/* CountingHashTable<Key, Value, ...>                                  */
/* ------------------------------------------------------------------ */

/* CountingHashTable(min_capacity, seed, max_count, no_init)
 * (counting_hash_table.cuh:75-85) */
int wc_counting_create(const wc_table_config *cfg, uint64_t min_capacity,
                       uint64_t seed, uint64_t max_count, int no_init,
                       wc_table **out);
/* insert(keys_in, num_in, stream, probing_length, status_out)
 * (counting_hash_table.cuh:184-194) */
int wc_counting_insert(wc_table *t, const void *keys_in, uint64_t num_in,
                       wc_stream_t stream, uint64_t probing_length,
                       void *status_out, int status_handler, uint32_t ignore);
/* retrieve(keys_in, num_in, values_out, stream, probing_length, status_out)
 * (counting_hash_table.cuh:238-249); counts clamped to max_count, written
 * on hits only */
int wc_counting_retrieve(wc_table *t, const void *keys_in, uint64_t num_in,
                         void *values_out, wc_stream_t stream,
                         uint64_t probing_length, void *status_out,
                         int status_handler, uint32_t ignore);
/* erase (counting_hash_table.cuh:292-301, with the stream passed through) */
int wc_counting_erase(wc_table *t, const void *keys_in, uint64_t num_in,
                      wc_stream_t stream, uint64_t probing_length,
                      void *status_out, int status_handler, uint32_t ignore);

/* ------------------------------------------------------------------ */
/* MultiValueHashTable<Key, Value, EmptyKey, TombstoneKey, ProbingScheme> */
/* (multi_value_hash_table.cuh); kind 3.  Every (key, value) pair takes  */
/* a slot of its own.  wc_svht_default_config gives the reference's     */
/* defaults.  size, init, retrieve_all (all pairs), peek/pop_status,    */
/* get_info and destroy are the wc_table_* calls.                        */
/* ------------------------------------------------------------------ */

/* MultiValueHashTable(min_capacity, seed, max_values_per_key, no_init)
 * (multi_value_hash_table.cuh:101-125) */
int wc_mvht_create(const wc_table_config *cfg, uint64_t min_capacity, uint64_t seed,
                   uint64_t max_values_per_key, int no_init, wc_table **out);
/* insert (:200-326): a key that already holds max_values_per_key values
 * reports duplicate_key + max_values_for_key_reached and is not stored; a
 * key that held values reports duplicate_key */
int wc_mvht_insert(wc_table *t, const void *keys_in, const void *values_in, uint64_t num_in,
                   wc_stream_t stream, uint64_t probing_length, void *status_out,
                   int status_handler, uint32_t ignore);
/* num_values (:769-800): values per key into num_per_key_out (device, may
 * be NULL) and their sum into *num_out (host); synchronises `stream` */
int wc_mvht_num_values(wc_table *t, const void *keys_in, uint64_t num_in, uint64_t *num_out,
                       uint64_t *num_per_key_out, wc_stream_t stream, uint64_t probing_length,
                       void *status_out, int status_handler, uint32_t ignore);
/* retrieve (:371-520): every key's values, in insertion order, at
 * values_out[begin_offsets_out[i] .. end_offsets_out[i]); *num_out (host)
 * gets the total.  With values_out NULL it is a dry run: end_offsets_out
 * gets the per-key counts (not summed), every status is dry_run.  The
 * offsets are uint64; synchronises `stream` before the values pass. */
int wc_mvht_retrieve(wc_table *t, const void *keys_in, uint64_t num_in,
                     uint64_t *begin_offsets_out, uint64_t *end_offsets_out, void *values_out,
                     uint64_t *num_out, wc_stream_t stream, uint64_t probing_length,
                     void *status_out, int status_handler, uint32_t ignore);
/* retrieve_all_keys (:561-598): each stored key once (order unspecified);
 * with keys_out NULL *num_out gets num_keys() (a dry run) */
int wc_mvht_retrieve_all_keys(wc_table *t, void *keys_out, uint64_t *num_out, wc_stream_t stream);
/* num_keys (:720-735): keys that hold at least one value */
int wc_mvht_num_keys(wc_table *t, wc_stream_t stream, uint64_t *out);

/* ------------------------------------------------------------------ */
/* Input generators (random_distributions.cuh:50-326), on the device.   */
/* Element i depends only on (seed, i): the same output for any launch  */
/* shape.  splitmix64 replaces the reference's kiss_rng (absent).       */
/* ------------------------------------------------------------------ */

/* uniform_distribution (:50-137): n uniform 4- or 8-byte words */
int wc_gen_uniform(void *out, uint64_t n, uint32_t bytes, uint64_t seed, wc_stream_t stream);
/* unique_distribution (:144-251): n distinct keys, never 0 or all ones
 * (the default empty and tombstone keys), at most 2^32 - 2 for 4-byte keys;
 * a bijection of the index where the reference rejects Bloom positives */
int wc_gen_unique(void *out, uint64_t n, uint32_t key_bytes, uint64_t seed, wc_stream_t stream);
/* zipf_distribution (:259-326): n_out draws of Zipf(s) over ranks
 * 1 .. n_in by the reference's rejection sampler; out gets in[rank - 1],
 * or the 1-based rank when `in` is NULL (the reference writes in[rank] and
 * rank + 1, one past the ranks).  s > 0 and s != 1. */
int wc_gen_zipf(const void *in, uint64_t n_in, void *out, uint64_t n_out, uint32_t bytes,
                double s, uint64_t seed, wc_stream_t stream);

/* ------------------------------------------------------------------ */
/* BucketListHashTable<Key, Value, EmptyKey, TombstoneKey,               */
/* BucketListStore<Value, IndexBits, CounterBits, SizeBits>, Probing>    */
/* (bucket_list_hash_table.cuh, storage.cuh:651-1454).  A key table maps */
/* each key to a list of value buckets in a pool of value_capacity       */
/* elements: the first bucket holds min_bucket_size values, each later   */
/* one a header and ceil(previous size * grow_factor) values, at most    */
/* max_bucket_size.  The bit widths bound the pool (2^index_bits - 1),   */
/* the values per key (2^counter_bits - 1) and the bucket size           */
/* (2^size_bits - 1); the reference's defaults are 32 / 20 / 10.         */
/* ------------------------------------------------------------------ */

typedef struct wc_blht wc_blht;

typedef struct wc_blht_info {
    uint32_t key_bytes, value_bytes, cg_size, probing, hasher1, hasher2;
    uint32_t index_bits, counter_bits, size_bits;
    float grow_factor;
    uint64_t key_capacity;    /* key slots, reference capacity rule */
    uint64_t value_capacity;  /* pool elements */
    uint64_t num_buckets;     /* key_capacity / cg_size */
    uint64_t seed, empty_key, tombstone_key;
    uint64_t min_bucket_size, max_bucket_size, max_values_per_key;
    uint64_t bytes_total;     /* keys, handles, pool, the pool counter */
    void *keys;               /* device: key_capacity keys */
    unsigned long long *handles; /* device: one list handle per key slot */
    unsigned long long *pool; /* device: value_capacity values or bucket headers */
    unsigned long long *next_free; /* device: pool elements handed out */
    uint32_t *status;         /* device Status word */
    int is_initialized;
} wc_blht_info;

/* BucketListHashTable(key_capacity, value_capacity, seed, grow_factor,
 * min_bucket_size, max_bucket_size, max_values_per_key, no_init)
 * (bucket_list_hash_table.cuh:106-121) with BucketListStore's bit widths;
 * a configuration the store refuses (storage.cuh:990-1014) is
 * WC_ERR_INVALID_ARGUMENT.  max_values_per_key is capped at
 * 2^counter_bits - 1. */
int wc_blht_create(const wc_table_config *cfg, uint64_t key_capacity, uint64_t value_capacity,
                   uint64_t seed, float grow_factor, uint64_t min_bucket_size,
                   uint64_t max_bucket_size, uint64_t max_values_per_key, uint32_t index_bits,
                   uint32_t counter_bits, uint32_t size_bits, int no_init, wc_blht **out);
int wc_blht_destroy(wc_blht *t);
/* init(seed) (:160-176): keys empty, every list empty, pool counter zero */
int wc_blht_init(wc_blht *t, uint64_t seed, wc_stream_t stream);
/* insert (:235-326): the key's status from the key table (none,
 * duplicate_key, probing_length_exceeded, invalid_key) plus the append's
 * (max_values_for_key_reached, out_of_memory when the pool is used up).
 * Every key gets a status; the reference writes none for a key that found
 * no slot. */
int wc_blht_insert(wc_blht *t, const void *keys_in, const void *values_in, uint64_t num_in,
                   wc_stream_t stream, uint64_t probing_length, void *status_out,
                   int status_handler, uint32_t ignore);
/* num_values (:776-800): list lengths per key and their sum (synchronises) */
int wc_blht_num_values(wc_blht *t, const void *keys_in, uint64_t num_in, uint64_t *num_out,
                       uint64_t *num_per_key_out, wc_stream_t stream, uint64_t probing_length,
                       void *status_out, int status_handler, uint32_t ignore);
/* retrieve (:375-466): every key's list at values_out[begin[i] .. end[i]),
 * newest bucket first; values_out NULL is a dry run (per-key counts in
 * end_offsets_out, status dry_run).  Synchronises `stream`. */
int wc_blht_retrieve(wc_blht *t, const void *keys_in, uint64_t num_in,
                     uint64_t *begin_offsets_out, uint64_t *end_offsets_out, void *values_out,
                     uint64_t *num_out, wc_stream_t stream, uint64_t probing_length,
                     void *status_out, int status_handler, uint32_t ignore);
/* retrieve_all_keys (:574-605): every stored key, order unspecified;
 * keys_out NULL gives the count */
int wc_blht_retrieve_all_keys(wc_blht *t, void *keys_out, uint64_t *num_out, wc_stream_t stream);
/* num_keys (:719-726), num_values() (:797-818: the sum of all list
 * lengths), the pool elements handed out (value_load_factor = used /
 * value_capacity, storage.cuh:1369-1396) */
int wc_blht_num_keys(wc_blht *t, wc_stream_t stream, uint64_t *out);
int wc_blht_total_values(wc_blht *t, wc_stream_t stream, uint64_t *out);
int wc_blht_pool_used(wc_blht *t, wc_stream_t stream, uint64_t *out);
int wc_blht_peek_status(wc_blht *t, wc_stream_t stream, uint32_t *out);
int wc_blht_pop_status(wc_blht *t, wc_stream_t stream, uint32_t *out);
int wc_blht_get_info(const wc_blht *t, wc_blht_info *info);

/* ------------------------------------------------------------------ */
/* MultiBucketHashTable<Key, Value, EmptyKey, TombstoneKey, EmptyValue,  */
/* ProbingScheme, AoSStore<Key, ArrayBucket<Value, B>>>                  */
/* (multi_bucket_hash_table.cuh).  A slot holds a key and a bucket of    */
/* B values (1 <= B <= cg_size); a key's values fill its last bucket     */
/* before the key takes another slot.  The config's key fields, probing  */
/* and cg_size are used as for the other tables; value_bytes (4 or 8) is */
/* independent of key_bytes.  Keys and buckets are stored as two arrays. */
/* ------------------------------------------------------------------ */

typedef struct wc_mbht wc_mbht;

typedef struct wc_mbht_info {
    uint32_t key_bytes, value_bytes, bucket_size, cg_size;
    uint32_t probing, hasher1, hasher2;
    uint64_t capacity;        /* key slots, reference capacity rule */
    uint64_t value_capacity;  /* capacity * bucket_size (:1088-1093) */
    uint64_t num_buckets;     /* capacity / cg_size */
    uint64_t seed, empty_key, tombstone_key, empty_value, max_values_per_key;
    uint64_t bytes_total;     /* bytes of this layout: keys, buckets, one index */
    void *keys;               /* device: capacity keys */
    void *values;             /* device: capacity * bucket_size values */
    uint32_t *status;         /* device Status word */
    unsigned long long *num_keys, *num_occupied; /* device counters */
    int is_initialized;
} wc_mbht_info;

/* MultiBucketHashTable(min_capacity, seed, max_values_per_key, no_init)
 * (multi_bucket_hash_table.cuh:195-217); bucket_size is ArrayBucket's B and
 * empty_value the EmptyValue parameter (default 0) */
int wc_mbht_create(const wc_table_config *cfg, uint32_t bucket_size, uint64_t empty_value,
                   uint64_t min_capacity, uint64_t seed, uint64_t max_values_per_key, int no_init,
                   wc_mbht **out);
int wc_mbht_destroy(wc_mbht *t);
/* init (:253-271): keys empty, bucket values empty, counters and status zero */
int wc_mbht_init(wc_mbht *t, wc_stream_t stream);
/* insert (:343-542): a key holding max_values_per_key values reports
 * duplicate_key + max_values_for_key_reached; an empty value reports
 * invalid_value; a key that held values reports duplicate_key */
int wc_mbht_insert(wc_mbht *t, const void *keys_in, const void *values_in, uint64_t num_in,
                   wc_stream_t stream, uint64_t probing_length, void *status_out,
                   int status_handler, uint32_t ignore);
/* num_values (:1013-1039): per key into num_per_key_out (device, may be
 * NULL), their sum into *num_out (host); synchronises `stream` */
int wc_mbht_num_values(wc_mbht *t, const void *keys_in, uint64_t num_in, uint64_t *num_out,
                       uint64_t *num_per_key_out, wc_stream_t stream, uint64_t probing_length,
                       void *status_out, int status_handler, uint32_t ignore);
/* retrieve (:574-680): every key's values at values_out[begin[i] .. end[i]),
 * in slot order along the probe sequence (insertion order); *num_out gets
 * the total.  values_out NULL is a dry run: end_offsets_out gets the
 * per-key counts, every status is dry_run.  Synchronises `stream`. */
int wc_mbht_retrieve(wc_mbht *t, const void *keys_in, uint64_t num_in,
                     uint64_t *begin_offsets_out, uint64_t *end_offsets_out, void *values_out,
                     uint64_t *num_out, wc_stream_t stream, uint64_t probing_length,
                     void *status_out, int status_handler, uint32_t ignore);
/* retrieve_all_keys (:742-777): each stored key once, order unspecified;
 * keys_out NULL gives num_keys() and joins dry_run */
int wc_mbht_retrieve_all_keys(wc_mbht *t, void *keys_out, uint64_t *num_out, wc_stream_t stream);
/* num_keys (:891-902), num_occupied (:904-916), size = num_values() (:1060-1082) */
int wc_mbht_num_keys(wc_mbht *t, wc_stream_t stream, uint64_t *out);
int wc_mbht_num_occupied(wc_mbht *t, wc_stream_t stream, uint64_t *out);
int wc_mbht_size(wc_mbht *t, wc_stream_t stream, uint64_t *out);
/* peek_status / pop_status (:1165-1201) */
int wc_mbht_peek_status(wc_mbht *t, wc_stream_t stream, uint32_t *out);
int wc_mbht_pop_status(wc_mbht *t, wc_stream_t stream, uint32_t *out);
int wc_mbht_get_info(const wc_mbht *t, wc_mbht_info *info);

/* ------------------------------------------------------------------ */
/* BloomFilter<Key, Hasher, Slot, CGSize>                               */
/* ------------------------------------------------------------------ */

typedef struct wc_bloom_config {
    uint32_t key_bytes;  /* 4 or 8 */
    uint32_t slot_bytes; /* 4 or 8 */
    uint32_t cg_size;    /* slots per block: 1, 2, 4, 8, 16 or 32 */
    uint32_t hasher;     /* WC_HASH_* */
} wc_bloom_config;

typedef struct wc_bloom_info {
    uint32_t key_bytes, slot_bytes, cg_size, hasher;
    uint64_t num_bits, num_slots, num_blocks, k, seed;
    void *words; /* device pointer to the bit vector (this filter's blocks) */
    uint64_t block_base, local_blocks; /* the blocks held: all, or a shard's */
} wc_bloom_info;

typedef struct wc_bloom wc_bloom;

/* BloomFilter(num_bits, k, seed) (bloom_filter.cuh:78-93) */
int wc_bloom_create(const wc_bloom_config *cfg, uint64_t num_bits, uint64_t k,
                    uint64_t seed, wc_bloom **out);
/* ~BloomFilter (bloom_filter.cuh:130-138) */
int wc_bloom_destroy(wc_bloom *b);
/* Sharded form (no counterpart in the reference, which is single-GPU):
 * shard `shard` of `num_shards` holds the blocks b of the whole filter
 * (num_bits, k, seed) with b * num_shards / num_blocks == shard, so each
 * block, and every bit a key sets, lives on one shard, and the shards'
 * words are the whole filter's words cut in block ranges.  Blocks of at most
 * 128 bytes and num_bits a multiple of the block bits.  A shard skips keys
 * of blocks it does not hold (query: absent).  wc_bloom_partition groups
 * keys by the shard that holds their block (counts_out: num_parts entries;
 * scratch: 2 * num_parts + 1 entries; perm_out: input position of each
 * output key), for the exchange step of a multi-GPU filter. */
int wc_bloom_create_shard(const wc_bloom_config *cfg, uint64_t num_bits, uint64_t k,
                          uint64_t seed, uint32_t shard, uint32_t num_shards, wc_bloom **out);
int wc_bloom_partition(const wc_bloom *b, const void *keys, uint64_t n, uint32_t num_parts,
                       void *keys_out, uint64_t *perm_out, uint64_t *counts_out,
                       uint64_t *scratch, wc_stream_t stream);
/* init(seed, stream) (bloom_filter.cuh:143-152) */
int wc_bloom_init(wc_bloom *b, uint64_t seed, wc_stream_t stream);
/* insert(keys_in, num_in, stream) (bloom_filter.cuh:200-208) */
int wc_bloom_insert(wc_bloom *b, const void *keys_in, uint64_t num_in,
                    wc_stream_t stream);
/* retrieve(keys_in, num_in, flags_out, stream) (bloom_filter.cuh:246-255) */
int wc_bloom_retrieve(wc_bloom *b, const void *keys_in, uint64_t num_in,
                      uint8_t *flags_out, wc_stream_t stream);
/* num_bits(), num_slots(), num_blocks(), k() and the device view */
int wc_bloom_get_info(const wc_bloom *b, wc_bloom_info *info);
/* fpr(n) (bloom_filter.cuh:342-354), the reference's own formula */
int wc_bloom_fpr(const wc_bloom *b, uint64_t n, double *out);

/* ------------------------------------------------------------------ */
/* Launch tuning (no counterpart in the reference, whose launches are    */
/* fixed at SDIV(n * cg, WARPCORE_BLOCKSIZE) x WARPCORE_BLOCKSIZE,       */
/* single_value_hash_table.cuh:255-257)                                  */
/* ------------------------------------------------------------------ */

/* ------------------------------------------------------------------ */
/* Bulk operations on host buffers (no counterpart in the reference,     */
/* whose bulk calls take device pointers only)                           */
/* ------------------------------------------------------------------ */

/* A pipe stages host buffers through `depth` device slots of `chunk_keys`
 * keys (0, 0: 2^22 keys, 3 slots; 16 bytes of device memory per staged
 * key) and owns a copy-in and a copy-out stream.  Chunk i's copy-in, chunk
 * i-1's kernel and chunk i-2's copy-out run at the same time.  Host
 * buffers should be pinned (cudaHostAlloc / cudaHostRegister) for copies to
 * overlap; pageable buffers work but copy synchronously.  One pipe serves
 * one call at a time. */
typedef struct wc_host_pipe wc_host_pipe;
int wc_host_pipe_create(uint64_t chunk_keys, uint32_t depth, wc_host_pipe **out);
int wc_host_pipe_destroy(wc_host_pipe *p);
/* Insert (single-value: keys and values; hash set: keys; counting: keys
 * counted) from host buffers.  Stream-ordered on `stream`: the copies start
 * after the caller's earlier work on `stream`, the kernels run on it, and
 * the host buffers must stay valid until `stream` passes the call. */
int wc_table_insert_host(wc_host_pipe *p, wc_table *t, const void *h_keys, const void *h_values,
                         uint64_t num_in, wc_stream_t stream, uint64_t probing_length);
/* Retrieve into a host buffer: values (single-value, counting) or one flag
 * byte per key (hash set).  Single-value and counting retrieves write hits
 * only, as the device call does: with miss_fill NULL a miss keeps the
 * output's content (copied in with the keys); otherwise a miss gets
 * *miss_fill (one value), which saves that copy.  The output is complete
 * once `stream` passes the call. */
int wc_table_retrieve_host(wc_host_pipe *p, wc_table *t, const void *h_keys, uint64_t num_in,
                           void *h_out, const void *miss_fill, wc_stream_t stream,
                           uint64_t probing_length);

/* ------------------------------------------------------------------ */
/* Fingerprints (no counterpart in the reference)                        */
/* ------------------------------------------------------------------ */

/* A table may keep one fingerprint byte per slot, so that probing reads a
 * bucket's cg_size bytes instead of its whole window and reads a slot only
 * where the fingerprint matches.  Results are the same either way.
 * AUTO (default): tables whose slot array is larger than L2; ALWAYS /
 * NEVER: every table.  Applies to tables created after the call.  The
 * environment variable WARPCORE_B200_FINGERPRINTS (auto, always, never)
 * sets the mode before the first call. */
#define WC_FINGERPRINTS_AUTO 0
#define WC_FINGERPRINTS_ALWAYS 1
#define WC_FINGERPRINTS_NEVER 2
int wc_fingerprint_policy(int mode, int *previous);
/* Which operations read fingerprints first on tables that have them: bit
 * 0 insert, 1 counting insert, 2 retrieve, 3 erase (default: all four;
 * an operation whose bit is clear probes whole windows and keeps the
 * fingerprints up to date).  Bit 4: a fingerprint-first insert loads the
 * slot it is about to claim before the compare-and-swap.  Bit 5: never
 * replace a large insert (more than 1/8 of a table whose fingerprints
 * exceed half of L2) by a whole-window insert without fingerprint writes
 * followed by a streaming rebuild of all fingerprints, which is the
 * default. */
int wc_fingerprint_ops(uint32_t op_mask, uint32_t *previous);
/* Which operations may probe whole windows with one key per lane (each
 * lane reads its key's window with 32-byte loads; bit 0 insert, 2 retrieve,
 * 3 erase, default all three) instead of with groups of lanes per window
 * and ballots.  Applies to tables whose slot array fits in L2 and whose
 * window is at most 128 bytes (64 bytes for inserts); counting inserts
 * (bit 1) always use the group kernel.  Results are the same either way. */
int wc_lane_ops(uint32_t op_mask, uint32_t *previous);

/* ------------------------------------------------------------------ */
/* Region passes (no counterpart in the reference)                       */
/* ------------------------------------------------------------------ */

/* Random reads on B200 slow down sharply once the array they hit outgrows
 * the GPU's address-translation reach (64-byte reads at random: 64 G/s over
 * 256 MiB, 13.5 G/s over 512 MiB).  A Bloom filter with blocks of at most
 * 128 bytes whose words exceed the region size of the operation is inserted
 * into (WC_REGION_INSERT) or queried (WC_REGION_QUERY) in passes, default
 * 256 MiB for both, each streaming all keys and serving those
 * whose block lies in one region of the filter.  0 = always one pass;
 * otherwise 1 MiB .. 1 TiB.  Applies to later calls (*previous gets the old
 * value).  Results do not depend on it. */
#define WC_REGION_INSERT 0
#define WC_REGION_QUERY 1
int wc_region_bytes(int op, uint64_t bytes, uint64_t *previous);

/* ------------------------------------------------------------------ */
/* L2 persistence for tables that fit in L2 (no counterpart in the       */
/* reference)                                                            */
/* ------------------------------------------------------------------ */

/* A table or filter whose slot array fits the device's persisting-L2
 * maximum (cudaDevAttrMaxPersistingL2CacheSize) launches its kernels with an
 * access-policy window over that array: its lines persist in L2 while keys
 * and outputs stream past, and while other work runs between calls.  Arrays
 * get windows at creation, in order, while the windows of all live arrays
 * on the device fit the persisting set-aside together; the others launch
 * without one.  The first such array sets this process's persisting-L2
 * limit once per device.  On by default (environment variable
 * WARPCORE_B200_L2_PERSIST=0 in the Python binding turns it off);
 * `enable` = 0 turns the windows off for later launches and creations
 * (*previous gets the old setting). */
int wc_l2_persistence(int enable, int *previous);
/* the window a table's launches use now: bytes (0 = none) and hit ratio */
int wc_table_l2_window(const wc_table *t, uint64_t *bytes_out, float *hit_ratio_out);

/* Buckets of the tuning table: load factor (inserted keys since init over
 * capacity) < 0.5, < 0.7, < 0.85, >= 0.85; batch size 2^(6+2b) .. 2^(8+2b). */
#define WC_TUNE_LOAD_BUCKETS 4
#define WC_TUNE_SIZE_BUCKETS 12
/* Launch geometry for (key width, op, load bucket, size bucket): threads
 * per block (multiple of 32, <= 256; 0 = default 256) and resident blocks
 * per SM (0 = occupancy limit).  op: 0 insert, 1 counting insert,
 * 2 retrieve, 3 erase.  Written by warpcore_b200.autotune. */
int wc_tune_set(uint32_t key_bytes, int op, uint32_t load_bucket, uint32_t size_bucket,
                uint32_t block_threads, uint32_t blocks_per_sm);
/* forget every tuned entry */
int wc_tune_reset(void);
/* Loads a tuning file written by `python -m warpcore_b200.autotune` (its
 * "entries": one wc_tune_set each).  path NULL: the environment variable
 * WARPCORE_B200_TUNING, else tuning_b200.json next to this library; "none"
 * loads nothing.  *loaded (if not NULL) gets the number of entries.  The
 * Python binding and the C++ class templates call it once. */
int wc_tune_load(const char *path, uint64_t *loaded);

/* ------------------------------------------------------------------ */
/* Batches: many requests on many tables in one launch                  */
/* (no counterpart in the reference, which launches one kernel per bulk */
/* call, single_value_hash_table.cuh:241-337)                            */
/* ------------------------------------------------------------------ */

#define WC_OP_INSERT 0
#define WC_OP_RETRIEVE 2

/* One request of a batch: the arguments of wc_svht_insert or
 * wc_svht_retrieve for one single-value table. */
typedef struct wc_batch_request {
    wc_table *table;
    int op;               /* WC_OP_INSERT or WC_OP_RETRIEVE */
    int status_handler;   /* WC_HANDLER_* */
    uint32_t ignore;      /* ReturnBoolean's Ignore */
    uint32_t reserved;
    const void *keys;     /* device, num keys */
    const void *values;   /* device, insert only */
    void *values_out;     /* device, retrieve only (written on hits) */
    void *status_out;     /* device or NULL */
    uint64_t num;
} wc_batch_request;

typedef struct wc_batch wc_batch;

/* A batch runner for up to max_requests requests per run.  It owns pinned
 * and device staging for `depth` runs in flight and one CUDA graph per
 * staging slot (a descriptor copy and the batch kernel), re-parameterised
 * for every run. */
int wc_batch_create(uint32_t max_requests, uint32_t depth, wc_batch **out);
int wc_batch_destroy(wc_batch *b);
/* Runs all requests in ONE kernel launch on `stream`, asynchronously.  All
 * tables must be single-value tables with the same key/value width and
 * cg_size.  The requests of one run must commute (different tables, or
 * requests of one kind on a table).  blocks_per_sm = 0 picks the occupancy
 * limit.  The caller keeps the request buffers alive until the stream has
 * passed the run; wc_batch_run blocks only when all `depth` staging slots
 * are still in flight. */
int wc_batch_run(wc_batch *b, const wc_batch_request *reqs, uint32_t num_requests,
                 wc_stream_t stream, uint64_t probing_length, uint32_t blocks_per_sm);

/* ------------------------------------------------------------------ */
/* Serving loop (no counterpart in the reference)                       */
/* ------------------------------------------------------------------ */

#define WC_SERVE_PLAIN 0
#define WC_SERVE_BATCHED 1
#define WC_SERVE_PERSISTENT 2

/* One timestamped request on a resident single-value table. */
typedef struct wc_serve_request {
    double arrival_us;    /* arrival time relative to the start of the run */
    wc_table *table;
    uint64_t table_id;    /* dense id of the table (0 .. number of tables) */
    int op;               /* WC_OP_INSERT or WC_OP_RETRIEVE */
    int reserved;
    const void *keys;     /* device */
    const void *values;   /* device, insert */
    void *values_out;     /* device, retrieve */
    uint64_t num;
} wc_serve_request;

typedef struct wc_serve_options {
    int mode;                    /* WC_SERVE_PLAIN, WC_SERVE_BATCHED or WC_SERVE_PERSISTENT */
    uint32_t streams;            /* streams (0: 4); plain: tables hashed onto them,
                                    batched: batches round-robin */
    uint32_t depth;              /* batched: batches in flight per stream (0: 2) */
    uint32_t max_batch_requests; /* batched: requests per batch (0: 4096) */
    uint64_t max_batch_keys;     /* batched: keys per batch (0: no limit);
                                    persistent: keys per chunk (0: 1024) */
    uint32_t blocks_per_sm;      /* batched: 0 = occupancy limit; persistent: 0 = 2 */
    uint32_t reserved;
    uint64_t probing_length;
    struct wc_table_pool *pool;  /* persistent only: requests name tables of this
                                    pool by table_id (their `table` is ignored)
                                    and are admitted against its budget; NULL:
                                    every request's table is resident */
} wc_serve_options;

typedef struct wc_serve_stats {
    uint64_t launches, batches, max_keys_in_batch;
    double host_wall_us;
    double gpu_batch_us;   /* batched: summed GPU time of the batches */
    double host_launch_us; /* batched: summed host time to launch them */
} wc_serve_stats;

/* ------------------------------------------------------------------ */
/* Table pool: tables admitted against a device-memory budget (no        */
/* counterpart in the reference)                                         */
/* ------------------------------------------------------------------ */

/* A set of single-value tables that share a device-memory budget.  A table
 * is registered (wc_table_pool_add) without device memory and becomes
 * resident when a request needs it: placed on memory of the pool's own
 * stream-ordered memory pool (wc_svht_create_on), new and initialised, or
 * restored from its host copy.  When the budget (resident tables plus the
 * buffers of requests in flight) has no room, the least recently used
 * tables with nothing in flight are copied to pinned host memory and their
 * device memory goes back to the pool.  Stream-ordered allocation
 * (cudaMallocAsync / cudaFreeAsync) never waits for the device, so tables
 * move while a persistent server runs. */
typedef struct wc_table_pool wc_table_pool;
typedef struct wc_table_pool_stats {
    uint64_t admissions;      /* tables placed in device memory */
    uint64_t restores;        /* of those, restored from a host copy */
    uint64_t evictions;       /* tables copied out to host memory */
    uint64_t waits;           /* requests that waited for budget */
    uint64_t peak_bytes;      /* highest resident + in-flight buffer bytes */
    uint64_t resident_bytes;  /* now */
    uint64_t resident_tables; /* now */
} wc_table_pool_stats;
int wc_table_pool_create(uint64_t budget_bytes, wc_table_pool **out);
/* registers a table (no device memory yet); *id_out is its table_id */
int wc_table_pool_add(wc_table_pool *p, const wc_table_config *cfg, uint64_t min_capacity,
                      uint64_t seed, uint64_t *id_out);
/* makes table `id` resident (evicting others if needed) and returns its
 * handle, valid until the pool moves it again */
int wc_table_pool_table(wc_table_pool *p, uint64_t id, wc_table **out);
int wc_table_pool_get_stats(const wc_table_pool *p, wc_table_pool_stats *out);
int wc_table_pool_destroy(wc_table_pool *p);

/* Replays `num_requests` requests, sorted by arrival, in real time in the
 * chosen form and writes each request's completion time (microseconds from
 * the start: device events, or for the persistent form the kernel's
 * %globaltimer stamp mapped onto the host clock) to complete_us[] and, if
 * not NULL, the time it was issued to issue_us[].  Every table sees its
 * requests in arrival order.  Blocks until all requests are complete. */
int wc_serve_run(const wc_serve_request *reqs, uint64_t num_requests,
                 const wc_serve_options *opt, double *issue_us, double *complete_us,
                 wc_serve_stats *stats);

/* ------------------------------------------------------------------ */
/* Persistent server (no counterpart in the reference, whose every bulk  */
/* call is a kernel launch, gpu_engine.cuh:203-262)                      */
/* ------------------------------------------------------------------ */

/* One resident kernel takes insert / retrieve requests on single-value
 * tables from a ring in mapped host memory: submitting a request is a few
 * host stores, with no kernel launch.  A dispatcher warp cuts each request
 * into chunks of chunk_keys keys; every other warp of the grid takes chunks
 * in order and probes them; the warp that finishes a request's last chunk
 * stamps its completion in host memory.  Requests in flight together must
 * commute (no insert and retrieve of one table at once); wc_serve_run with
 * WC_SERVE_PERSISTENT keeps to that.  The kernel ends when the server is
 * stopped, or on its own after idle_timeout_us without a request; every
 * device-side wait is bounded.  The stream must be a non-blocking stream of
 * its own: the kernel occupies it until the stop.  Do not free device
 * memory (cudaFree synchronises the device) while a server runs. */
typedef struct wc_pserver wc_pserver;
typedef struct wc_pserver_options {
    uint32_t key_bytes;        /* 4 (u32/u32 tables) or 8 (u64/u64) */
    uint32_t cg_size;          /* window width of the tables served */
    uint32_t blocks_per_sm;    /* resident blocks of 256 threads (0: 2) */
    uint32_t reserved;
    uint64_t chunk_keys;       /* keys per chunk (0: 1024) */
    uint64_t idle_timeout_us;  /* 0: 2 s */
    uint64_t probing_length;
} wc_pserver_options;
/* launches the kernel on `stream` and returns once it runs */
int wc_pserver_start(const wc_pserver_options *opt, wc_stream_t stream, wc_pserver **out);
/* queues one request (device buffers; `values` for inserts, `values_out`
 * for retrieves, written on hits only); *ticket_out identifies it.  Waits
 * only if the ring's 4096 slots are all in flight. */
int wc_pserver_submit(wc_pserver *s, wc_table *table, int op, const void *keys,
                      const void *values, void *values_out, uint64_t num,
                      uint64_t *ticket_out);
/* *done = 1 once the request is complete; *complete_us (if not NULL) gets
 * its completion time on the server's host clock (wc_pserver_now_us) */
int wc_pserver_poll(wc_pserver *s, uint64_t ticket, int *done, double *complete_us);
int wc_pserver_now_us(const wc_pserver *s, double *now_us);
/* stops the kernel, waits for it and frees the server; WC_ERR_TIMEOUT if
 * the kernel had ended on a bounded wait (its idle limit) */
int wc_pserver_stop(wc_pserver *s);

/* ------------------------------------------------------------------ */
/* Key routing for tables sharded over GPUs (no counterpart in the       */
/* reference, which is single-GPU)                                       */
/* ------------------------------------------------------------------ */

#define WC_PARTITION_MAX_PARTS 1024

/* Groups keys (and values, if not NULL) by owning shard:
 * owner(key) = (hi32(fmix64(key ^ salt)) * num_parts) >> 32.  Writes the
 * grouped keys/values, perm_out[j] = input position of output j, and
 * counts_out[p] = keys owned by shard p (all device buffers; counts_out is
 * num_parts uint64, scratch is 2 * num_parts + 1 uint64).  Asynchronous on
 * `stream`.  The kernels check every output position against n; after the
 * stream completes, scratch[2 * num_parts] holds the number of keys that
 * failed the check and were dropped (0 unless the inputs changed while the
 * call ran). */
int wc_partition(const void *keys, const void *values, uint64_t n, uint32_t key_bytes,
                 uint32_t value_bytes, uint32_t num_parts, uint64_t salt, void *keys_out,
                 void *values_out, uint64_t *perm_out, uint64_t *counts_out,
                 uint64_t *scratch, wc_stream_t stream);
/* The inverse step of a sharded retrieve: answer j, in the order
 * wc_partition produced, goes back to input position perm[j].  Its value is
 * written only if status[j] is 0 (a hit), as retrieve writes hits only, or
 * always if status is NULL (Bloom flags); the status is written if
 * status_out is not NULL.  value_bytes 1 (flags), 4 or 8.  Entries whose
 * perm[j] is not below n are skipped.  Asynchronous on `stream`. */
int wc_partition_restore(const void *values, const uint32_t *status, const uint64_t *perm,
                         uint64_t n, uint32_t value_bytes, void *values_out,
                         uint32_t *status_out, wc_stream_t stream);

/* ------------------------------------------------------------------ */
/* Counting without allocating                                          */
/* ------------------------------------------------------------------ */

/* Largest slot array wc_slots_size_noalloc accepts (2^34 slots). */
#define WC_NOALLOC_MAX_SLOTS (1ull << 34)

/* No counterpart in the reference.  Counts the occupied slots (key neither
 * empty_key nor tombstone_key) of a slot array in this library's layout
 * (key_bytes 4 or 8; value_bytes 0 for a hash set, else equal to key_bytes)
 * and writes the count to *size_out, a DEVICE pointer to one uint64, on
 * `stream`, without allocating any device memory.  A key-only array (a hash
 * set's slots, the key array of a struct-of-arrays single-value table, or
 * the separate key array of a multi-bucket or bucket-list table, whose
 * wc_table_info reports value_bytes equal to key_bytes) must be
 * passed with value_bytes 0: the 8- or 16-byte key+value layout would count
 * it wrongly.  It is meant for callers
 * that hold a table's slots without a handle of this library and may not
 * allocate: e.g. a process that received the table's memory through CUDA
 * IPC, or a plugin whose host framework owns all device memory.  Scratch is
 * a fixed 512 KiB array inside the library (held by every GPU that loads
 * it); slot arrays above WC_NOALLOC_MAX_SLOTS are rejected with
 * WC_ERR_INVALID_ARGUMENT.  All calls share that array, so calls that
 * overlap on the GPU race.  Every call looks the array's address up in the
 * current context (the first call on a device loads it there and should come
 * before any stream capture).  `slots` must
 * be 16-byte aligned (wc_table_get_info's `slots` is). */
int wc_slots_size_noalloc(const void *slots, uint64_t capacity, uint32_t key_bytes,
                          uint32_t value_bytes, uint64_t empty_key,
                          uint64_t tombstone_key, wc_stream_t stream,
                          uint64_t *size_out);

#ifdef __cplusplus
}
#endif

#endif /* WARPCORE_B200_H */
