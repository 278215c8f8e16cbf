/*
 * wc_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of warpcore's hot
 * path, used as the checker for the CUDA library.  Every function cites the
 * reference file:line it follows (paths relative to the warpcore project).
 * See wc_oracle.h for the parity pin.
 */
#define _GNU_SOURCE
#include "wc_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------------ */
/* hashers (hashers.cuh:34-44 NvidiaHash, :70-77 MuellerHash,
 *          :116-124 fmix32, :131-139 fmix64, :147-175 IdentityMap)          */
/* ------------------------------------------------------------------------ */

static uint32_t fmix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

static uint64_t fmix64(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

static uint32_t nvidia32(uint32_t x)
{
    x = (x + 0x7ed55d16u) + (x << 12);
    x = (x ^ 0xc761c23cu) ^ (x >> 19);
    x = (x + 0x165667b1u) + (x << 5);
    x = (x + 0xd3a2646cu) ^ (x << 9);
    x = (x + 0xfd7046c5u) + (x << 3);
    x = (x ^ 0xb55a4f09u) ^ (x >> 16);
    return x;
}

static uint32_t mueller32(uint32_t x)
{
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x);
    return x;
}

static uint64_t kmask(int key_bytes)
{
    return key_bytes == 4 ? 0xffffffffull : ~0ull;
}

int wco_hash_bits(int hasher, int key_bytes)
{
    switch (hasher) {
    case WCO_HASH_MURMUR: return key_bytes * 8;
    case WCO_HASH_NVIDIA:
    case WCO_HASH_MUELLER:
    case WCO_HASH_IDENTITY32: return 32;
    default: return 64;
    }
}

uint64_t wco_hash(int hasher, int key_bytes, uint64_t x)
{
    x &= kmask(key_bytes);
    switch (hasher) {
    case WCO_HASH_MURMUR:
        return key_bytes == 4 ? (uint64_t)fmix32((uint32_t)x) : fmix64(x);
    case WCO_HASH_NVIDIA: return nvidia32((uint32_t)x);
    case WCO_HASH_MUELLER: return mueller32((uint32_t)x);
    case WCO_HASH_IDENTITY32: return (uint32_t)x;
    default: return x;
    }
}

/* ------------------------------------------------------------------------ */
/* prime chain (utils/generate_primes_hpp.py:20-43, defaults :70-73):
 * p0 = first prime >= 131072, p[i+1] = first prime >= p[i] + 131072,
 * up to 17177772037.  Computed here with a deterministic Miller-Rabin.     */
/* ------------------------------------------------------------------------ */

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m)
{
    return (uint64_t)((unsigned __int128)a * b % m);
}

static uint64_t powmod(uint64_t a, uint64_t e, uint64_t m)
{
    uint64_t r = 1;
    a %= m;
    while (e) {
        if (e & 1) r = mulmod(r, a, m);
        a = mulmod(a, a, m);
        e >>= 1;
    }
    return r;
}

static int is_prime_u64(uint64_t n)
{
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; i++) {
        if (n == small[i]) return 1;
        if (n % small[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; s++; }
    for (int i = 0; i < 12; i++) {
        uint64_t x = powmod(small[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int comp = 1;
        for (int r = 1; r < s; r++) {
            x = mulmod(x, x, n);
            if (x == n - 1) { comp = 0; break; }
        }
        if (comp) return 0;
    }
    return 1;
}

#define PRIME_STEP 131072ull
#define PRIME_MAX 17177772037ull

static uint64_t *g_primes = NULL;
static uint64_t g_num_primes = 0;
static pthread_once_t g_primes_once = PTHREAD_ONCE_INIT;

static void build_primes(void)
{
    uint64_t cap = 140000;
    uint64_t *p = (uint64_t *)malloc(cap * sizeof(uint64_t));
    uint64_t n = 0;
    uint64_t x = PRIME_STEP;
    for (;;) {
        while (!is_prime_u64(x)) x++;
        if (x > PRIME_MAX) break;
        p[n++] = x;
        x += PRIME_STEP;
    }
    g_primes = p;
    g_num_primes = n;
}

uint64_t wco_num_primes(void)
{
    pthread_once(&g_primes_once, build_primes);
    return g_num_primes;
}

void wco_primes(uint64_t *out)
{
    pthread_once(&g_primes_once, build_primes);
    memcpy(out, g_primes, g_num_primes * sizeof(uint64_t));
}

/* base.cuh:27-34: smallest table prime >= ceil(min/cg), times cg; 0 if none */
uint64_t wco_valid_capacity(uint64_t min_capacity, uint64_t cg_size)
{
    pthread_once(&g_primes_once, build_primes);
    uint64_t x = (min_capacity + cg_size - 1) / cg_size;
    uint64_t lo = 0, hi = g_num_primes;
    while (lo < hi) {
        uint64_t mid = (lo + hi) / 2;
        if (g_primes[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo == g_num_primes ? 0 : g_primes[lo] * cg_size;
}

/* ------------------------------------------------------------------------ */
/* probing iterators (probing_schemes.cuh:79-100 DoubleHashing,
 * LinearProbing begin/next, QuadraticProbing begin/next).
 * All lanes of a cooperative group advance together; lane r's slot is
 * pos[r].  The hash plus lane rank wraps in the hasher's output width,
 * because thread_block_tile::thread_rank() is an unsigned int.             */
/* ------------------------------------------------------------------------ */

typedef struct {
    int scheme, h1, h2, key_bytes;
    uint64_t cg, capacity, windows_left, base, step;
    uint64_t pos[32];
} probe_t;

static uint64_t wrap_add(uint64_t h, uint64_t r, int bits)
{
    uint64_t s = h + r;
    return bits == 32 ? (s & 0xffffffffull) : s;
}

/* number of windows the reference visits for a probing length:
 * SDIV(pl, cg) * cg slots per lane (probing_schemes.cuh:61), computed with
 * the same unsigned wrap; the first window is always visited. */
static uint64_t windows_for(uint64_t probing_length, uint64_t cg)
{
    uint64_t pl = (probing_length + cg - 1) / cg;
    return pl == 0 ? 1 : pl;
}

static void probe_begin(probe_t *p, int scheme, int h1, int h2, int key_bytes,
                        uint64_t cg, uint64_t capacity, uint64_t key,
                        uint64_t seed, uint64_t probing_length)
{
    const uint64_t km = kmask(key_bytes);
    p->scheme = scheme; p->h1 = h1; p->h2 = h2; p->key_bytes = key_bytes;
    p->cg = cg; p->capacity = capacity;
    p->windows_left = windows_for(probing_length, cg);
    const uint64_t h = wco_hash(h1, key_bytes, (key + seed) & km);
    const int hb = wco_hash_bits(h1, key_bytes);
    for (uint64_t r = 0; r < cg; r++) p->pos[r] = wrap_add(h, r, hb) % capacity;
    p->step = 1;
    p->base = 0;
    if (scheme == WCO_PROBE_DOUBLE) {
        const uint64_t h2v = wco_hash(h2, key_bytes, (key + seed + 1) & km);
        p->base = (h2v % (capacity / cg - 1) + 1) * cg;
    }
}

/* returns 0 when the sequence has ended */
static int probe_next(probe_t *p)
{
    if (p->windows_left <= 1) return 0;
    p->windows_left--;
    for (uint64_t r = 0; r < p->cg; r++) {
        if (p->scheme == WCO_PROBE_DOUBLE)
            p->pos[r] = (p->pos[r] + p->base) % p->capacity;
        else if (p->scheme == WCO_PROBE_LINEAR)
            p->pos[r] = (p->pos[r] + p->cg) % p->capacity;
        else
            p->pos[r] = (p->pos[r] + p->step) % p->capacity;
    }
    if (p->scheme == WCO_PROBE_QUADRATIC) p->step++;
    return 1;
}

uint64_t wco_probe_sequence(int scheme, int h1, int h2, int key_bytes,
                            uint64_t cg, uint64_t capacity, uint64_t key,
                            uint64_t seed, uint64_t probing_length,
                            uint64_t max_windows, uint64_t *out)
{
    probe_t p;
    probe_begin(&p, scheme, h1, h2, key_bytes, cg, capacity, key, seed,
                probing_length);
    uint64_t w = 0;
    do {
        if (w >= max_windows) break;
        for (uint64_t r = 0; r < cg; r++) out[w * cg + r] = p.pos[r];
        w++;
    } while (probe_next(&p));
    return w;
}

/* status.cuh:142-146 (operator~) and :316-330 (ReturnBoolean::handle):
 * ~Status(x) is (~x) ^ 0xFFF, so the flag is set for bits of the status
 * that are in Ignore's low twelve bits or at bit 12 and above. */
uint8_t wco_status_to_bool(uint32_t status, uint32_t ignore)
{
    const uint32_t m = (~ignore) ^ 0xFFFu;
    return (status & m) != 0;
}

/* ------------------------------------------------------------------------ */
/* tables: single_value_hash_table.cuh, hash_set.cuh, counting_hash_table.cuh */
/* ------------------------------------------------------------------------ */

struct wco_table {
    int kind, key_bytes, value_bytes, scheme, h1, h2;
    uint64_t capacity, cg, seed, empty, tomb, max_count;
    uint64_t *keys;
    uint64_t *values;
    uint32_t status;
    uint64_t max_values, num_keys; /* multi-value tables */
};

wco_table *wco_table_create(int kind, int key_bytes, int value_bytes,
                            uint64_t min_capacity, uint64_t seed, uint64_t cg,
                            int scheme, int h1, int h2, uint64_t empty_key,
                            uint64_t tombstone_key, uint64_t max_count)
{
    wco_table *t = (wco_table *)calloc(1, sizeof(wco_table));
    t->kind = kind;
    t->key_bytes = key_bytes;
    t->value_bytes = kind == WCO_HASHSET ? 0 : value_bytes;
    t->scheme = scheme; t->h1 = h1; t->h2 = h2;
    t->cg = cg;
    t->capacity = wco_valid_capacity(min_capacity, cg);
    t->empty = empty_key & kmask(key_bytes);
    t->tomb = tombstone_key & kmask(key_bytes);
    t->max_count = max_count;
    t->keys = (uint64_t *)malloc((t->capacity ? t->capacity : 1) * 8);
    t->values = (uint64_t *)calloc(t->capacity ? t->capacity : 1, 8);
    wco_table_init(t, seed);
    return t;
}

void wco_table_destroy(wco_table *t)
{
    if (!t) return;
    free(t->keys);
    free(t->values);
    free(t);
}

uint64_t wco_table_capacity(const wco_table *t) { return t->capacity; }

/* init(): keys := empty (storage.cuh:523-539); counting also zeroes the
 * values (counting_hash_table.cuh:114-124).  Values of a plain SVHT are
 * left as they were, like the reference. */
void wco_table_init(wco_table *t, uint64_t seed)
{
    t->seed = seed & kmask(t->key_bytes);
    for (uint64_t i = 0; i < t->capacity; i++) t->keys[i] = t->empty;
    if (t->kind == WCO_COUNTING)
        memset(t->values, 0, t->capacity * 8);
    t->status = 0;
    t->num_keys = 0;
}

static uint64_t load_elem(const void *p, int bytes, uint64_t i)
{
    return bytes == 4 ? ((const uint32_t *)p)[i] : ((const uint64_t *)p)[i];
}

static void store_elem(void *p, int bytes, uint64_t i, uint64_t v)
{
    if (bytes == 4) ((uint32_t *)p)[i] = (uint32_t)v;
    else ((uint64_t *)p)[i] = v;
}

static int valid_key(const wco_table *t, uint64_t k)
{
    return k != t->empty && k != t->tomb;
}

/* Status::atomic_join (status.cuh:187-193) */
static void join(wco_table *t, uint32_t s) { t->status |= s; }

/* insert_impl (single_value_hash_table.cuh:743-823; hash_set.cuh:193-254):
 * returns the slot index that holds the key afterwards, or -1. */
static int64_t insert_impl(wco_table *t, uint64_t key, uint64_t pl,
                           uint32_t *st)
{
    if (!valid_key(t, key)) {
        join(t, WCO_ST_INVALID_KEY);
        *st = WCO_ST_INVALID_KEY;
        return -1;
    }
    probe_t p;
    probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg, t->capacity,
                key, t->seed, pl);
    /* a cycle-free sequence has seen every slot after capacity/cg windows;
     * stop there instead of spinning like the unbounded reference loop */
    uint64_t guard = t->capacity / t->cg + 1;
    do {
        for (uint64_t r = 0; r < t->cg; r++) {
            if (t->keys[p.pos[r]] == key) {
                join(t, WCO_ST_DUPLICATE_KEY);
                *st = WCO_ST_DUPLICATE_KEY;
                return (int64_t)p.pos[r];
            }
        }
        for (uint64_t r = 0; r < t->cg; r++) {
            if (t->keys[p.pos[r]] == t->empty) {
                t->keys[p.pos[r]] = key;
                *st = WCO_ST_NONE;
                return (int64_t)p.pos[r];
            }
        }
    } while (--guard && probe_next(&p));
    join(t, WCO_ST_PROBING_LENGTH_EXCEEDED);
    *st = WCO_ST_PROBING_LENGTH_EXCEEDED;
    return -1;
}

void wco_insert(wco_table *t, const void *keys, const void *values, uint64_t n,
                uint64_t probing_length, uint32_t *status_out)
{
    const uint64_t vmask = t->value_bytes == 4 ? 0xffffffffull : ~0ull;
    for (uint64_t i = 0; i < n; i++) {
        uint32_t st = WCO_ST_UNKNOWN_ERROR;
        const uint64_t key = load_elem(keys, t->key_bytes, i);
        const int64_t slot = insert_impl(t, key, probing_length, &st);
        if (slot >= 0) {
            if (t->kind == WCO_SVHT) {
                /* single_value_hash_table.cuh:222-225 */
                t->values[slot] = load_elem(values, t->value_bytes, i);
            } else if (t->kind == WCO_COUNTING) {
                /* counting_hash_table.cuh:152-169 */
                uint64_t *v = &t->values[slot];
                if (*v < t->max_count) {
                    const uint64_t old = *v;
                    *v = (*v + 1) & vmask;
                    if (old > *v) {
                        st |= WCO_ST_INDEX_OVERFLOW;
                        join(t, WCO_ST_INDEX_OVERFLOW);
                        *v = t->max_count;
                    }
                }
            }
        }
        if (status_out) status_out[i] = st;
    }
}

/* SVHT::retrieve (single_value_hash_table.cuh:268-307), HashSet::retrieve
 * (hash_set.cuh:292-329), CountingHashTable::retrieve (:204-225), and the
 * kernel's hit-only write (gpu_engine.cuh:252-257). */
void wco_retrieve(wco_table *t, const void *keys, uint64_t n, void *values_out,
                  uint64_t probing_length, uint32_t *status_out)
{
    for (uint64_t i = 0; i < n; i++) {
        const uint64_t key = load_elem(keys, t->key_bytes, i);
        uint32_t st;
        uint64_t val = 0;
        int flag = 0;
        if (!valid_key(t, key)) {
            join(t, WCO_ST_INVALID_KEY);
            st = WCO_ST_INVALID_KEY;
        } else {
            probe_t p;
            probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg,
                        t->capacity, key, t->seed, probing_length);
            uint64_t guard = t->capacity / t->cg + 1;
            st = WCO_ST_PROBING_LENGTH_EXCEEDED;
            int done = 0;
            do {
                for (uint64_t r = 0; r < t->cg && !done; r++) {
                    if (t->keys[p.pos[r]] == key) {
                        val = t->values[p.pos[r]];
                        flag = 1;
                        st = WCO_ST_NONE;
                        done = 1;
                    }
                }
                if (done) break;
                for (uint64_t r = 0; r < t->cg && !done; r++) {
                    if (t->keys[p.pos[r]] == t->empty) {
                        done = 1;
                        flag = 0;
                        if (t->kind == WCO_HASHSET) {
                            st = WCO_ST_NONE;
                        } else {
                            st = WCO_ST_KEY_NOT_FOUND;
                            join(t, WCO_ST_KEY_NOT_FOUND);
                        }
                    }
                }
                if (done) break;
            } while (--guard && probe_next(&p));
            if (!done) join(t, WCO_ST_PROBING_LENGTH_EXCEEDED);
        }
        if (st == WCO_ST_NONE) {
            if (t->kind == WCO_HASHSET) {
                ((uint8_t *)values_out)[i] = (uint8_t)flag;
            } else {
                if (t->kind == WCO_COUNTING && val > t->max_count)
                    val = t->max_count;
                store_elem(values_out, t->value_bytes, i, val);
            }
        }
        if (status_out) status_out[i] = st;
    }
}

/* SVHT::erase (single_value_hash_table.cuh:426-468) and HashSet::erase
 * (hash_set.cuh:396-438, which always reports none). */
void wco_erase(wco_table *t, const void *keys, uint64_t n,
               uint64_t probing_length, uint32_t *status_out)
{
    for (uint64_t i = 0; i < n; i++) {
        const uint64_t key = load_elem(keys, t->key_bytes, i);
        uint32_t st;
        if (!valid_key(t, key)) {
            join(t, WCO_ST_INVALID_KEY);
            st = WCO_ST_INVALID_KEY;
        } else {
            probe_t p;
            probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg,
                        t->capacity, key, t->seed, probing_length);
            uint64_t guard = t->capacity / t->cg + 1;
            st = WCO_ST_PROBING_LENGTH_EXCEEDED;
            int done = 0;
            do {
                for (uint64_t r = 0; r < t->cg && !done; r++) {
                    if (t->keys[p.pos[r]] == key) {
                        t->keys[p.pos[r]] = t->tomb;
                        st = WCO_ST_NONE;
                        done = 1;
                    }
                }
                if (done) break;
                for (uint64_t r = 0; r < t->cg && !done; r++) {
                    if (t->keys[p.pos[r]] == t->empty) {
                        st = WCO_ST_KEY_NOT_FOUND;
                        done = 1;
                    }
                }
                if (done) break;
            } while (--guard && probe_next(&p));
            if (t->kind == WCO_HASHSET) st = WCO_ST_NONE;
        }
        if (status_out) status_out[i] = st;
    }
}

/* size() (single_value_hash_table.cuh:535-592, hash_set.cuh:500-557) */
uint64_t wco_size(const wco_table *t)
{
    uint64_t n = 0;
    for (uint64_t i = 0; i < t->capacity; i++) n += valid_key(t, t->keys[i]);
    return n;
}

/* retrieve_all (single_value_hash_table.cuh:391-417), in slot order */
uint64_t wco_retrieve_all(const wco_table *t, void *keys_out, void *values_out)
{
    uint64_t n = 0;
    for (uint64_t i = 0; i < t->capacity; i++) {
        if (!valid_key(t, t->keys[i])) continue;
        if (keys_out) store_elem(keys_out, t->key_bytes, n, t->keys[i]);
        if (values_out && t->value_bytes)
            store_elem(values_out, t->value_bytes, n, t->values[i]);
        n++;
    }
    return n;
}

uint32_t wco_peek_status(const wco_table *t) { return t->status; }

uint32_t wco_pop_status(wco_table *t)
{
    uint32_t s = t->status;
    t->status = 0;
    return s;
}

void wco_table_slots(const wco_table *t, uint64_t *keys_out,
                     uint64_t *values_out)
{
    if (keys_out) memcpy(keys_out, t->keys, t->capacity * 8);
    if (values_out) memcpy(values_out, t->values, t->capacity * 8);
}

/* ------------------------------------------------------------------------ */
/* MultiValueHashTable (multi_value_hash_table.cuh): every (key, value) pair  */
/* takes a slot of its own.                                                   */
/* ------------------------------------------------------------------------ */

wco_table *wco_mv_create(int key_bytes, int value_bytes, uint64_t min_capacity, uint64_t seed,
                         uint64_t cg, int scheme, int h1, int h2, uint64_t empty_key,
                         uint64_t tombstone_key, uint64_t max_values_per_key)
{
    wco_table *t = wco_table_create(WCO_SVHT, key_bytes, value_bytes, min_capacity, seed, cg,
                                    scheme, h1, h2, empty_key, tombstone_key, ~0ull);
    t->kind = WCO_MULTIVALUE;
    t->max_values = max_values_per_key;
    return t;
}

/* insert (multi_value_hash_table.cuh:200-289): along the probe sequence,
 * count the key's values window by window; stop with duplicate_key +
 * max_values_for_key_reached once the count reaches max_values_per_key;
 * otherwise claim the window's first empty slot (lane order).  A key that
 * had no value yet counts as a new key.  The status is duplicate_key when
 * the key had values (not joined on success). */
void wco_mv_insert(wco_table *t, const void *keys, const void *values, uint64_t n,
                   uint64_t probing_length, uint32_t *status_out)
{
    for (uint64_t i = 0; i < n; i++) {
        const uint64_t key = load_elem(keys, t->key_bytes, i);
        uint32_t st;
        if (!valid_key(t, key)) {
            join(t, WCO_ST_INVALID_KEY);
            st = WCO_ST_INVALID_KEY;
        } else {
            probe_t p;
            probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg, t->capacity, key,
                        t->seed, probing_length);
            uint64_t num = 0, guard = t->capacity / t->cg + 1;
            int done = 0;
            st = WCO_ST_PROBING_LENGTH_EXCEEDED;
            do {
                for (uint64_t r = 0; r < t->cg; r++) num += t->keys[p.pos[r]] == key;
                if (num >= t->max_values) {
                    st = WCO_ST_DUPLICATE_KEY | WCO_ST_MAX_VALUES_REACHED;
                    join(t, st);
                    done = 1;
                    break;
                }
                for (uint64_t r = 0; r < t->cg; r++) {
                    if (t->keys[p.pos[r]] == t->empty) {
                        t->keys[p.pos[r]] = key;
                        t->values[p.pos[r]] = load_elem(values, t->value_bytes, i);
                        if (num == 0) t->num_keys++;
                        st = num > 0 ? WCO_ST_DUPLICATE_KEY : WCO_ST_NONE;
                        done = 1;
                        break;
                    }
                }
                if (done) break;
            } while (--guard && probe_next(&p));
            if (!done) {
                st = WCO_ST_PROBING_LENGTH_EXCEEDED | (num > 0 ? WCO_ST_DUPLICATE_KEY : 0);
                join(t, st);
            }
        }
        if (status_out) status_out[i] = st;
    }
}

/* for_each over one key's values (multi_value_hash_table.cuh:607-663):
 * windows of the probe sequence (probing length capped at the capacity),
 * hits in lane order, until a window holds an empty slot or the count
 * reaches max_values_per_key.  Writes the values to out (if not NULL) and
 * returns the status; *num gets the count. */
static uint32_t mv_for_each(wco_table *t, uint64_t key, uint64_t probing_length, void *out,
                            uint64_t *num_out)
{
    if (!valid_key(t, key)) {
        *num_out = 0;
        join(t, WCO_ST_INVALID_KEY);
        return WCO_ST_INVALID_KEY;
    }
    probe_t p;
    const uint64_t pl = probing_length < t->capacity ? probing_length : t->capacity;
    probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg, t->capacity, key, t->seed,
                pl);
    uint64_t num = 0, guard = t->capacity / t->cg + 1;
    do {
        int any_empty = 0;
        for (uint64_t r = 0; r < t->cg; r++) {
            const uint64_t k = t->keys[p.pos[r]];
            if (k == key) {
                if (out) store_elem(out, t->value_bytes, num, t->values[p.pos[r]]);
                num++;
            }
            any_empty |= k == t->empty;
        }
        if (any_empty || num >= t->max_values) {
            *num_out = num;
            if (num == 0) {
                join(t, WCO_ST_KEY_NOT_FOUND);
                return WCO_ST_KEY_NOT_FOUND;
            }
            return WCO_ST_NONE;
        }
    } while (--guard && probe_next(&p));
    *num_out = num;
    join(t, WCO_ST_PROBING_LENGTH_EXCEEDED);
    return WCO_ST_PROBING_LENGTH_EXCEEDED;
}

/* bulk num_values (multi_value_hash_table.cuh:769-800, gpu_engine.cuh:467-501) */
uint64_t wco_mv_num_values(wco_table *t, const void *keys, uint64_t n, uint64_t *counts_out,
                           uint64_t probing_length, uint32_t *status_out)
{
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t num = 0;
        const uint32_t st = mv_for_each(t, load_elem(keys, t->key_bytes, i), probing_length,
                                        NULL, &num);
        if (counts_out) counts_out[i] = num;
        total += num;
        if (status_out) status_out[i] = st;
    }
    return total;
}

/* bulk retrieve (multi_value_hash_table.cuh:371-520, gpu_engine.cuh:305-346):
 * counts per key, an inclusive scan into end offsets, begin offsets one
 * behind, then every key's values in probe order at its begin offset.
 * With values_out NULL it is a dry run: end_offsets get the per-key counts
 * (not scanned) and every status is dry_run. */
uint64_t wco_mv_retrieve(wco_table *t, const void *keys, uint64_t n, uint64_t *begin_out,
                         uint64_t *end_out, void *values_out, uint64_t probing_length,
                         uint32_t *status_out)
{
    const uint64_t total = wco_mv_num_values(t, keys, n, end_out, probing_length, NULL);
    if (!values_out) {
        for (uint64_t i = 0; i < n && status_out; i++) status_out[i] = WCO_ST_DRY_RUN;
        join(t, WCO_ST_DRY_RUN);
        return total;
    }
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; i++) {
        begin_out[i] = s;
        s += end_out[i];
        end_out[i] = s;
    }
    for (uint64_t i = 0; i < n; i++) {
        uint64_t num = 0;
        char *dst = (char *)values_out + begin_out[i] * (uint64_t)t->value_bytes;
        uint32_t st = mv_for_each(t, load_elem(keys, t->key_bytes, i), probing_length, dst, &num);
        if (num != end_out[i] - begin_out[i]) {
            join(t, WCO_ST_INVALID_PHASE_OVERLAP);
            st |= WCO_ST_INVALID_PHASE_OVERLAP;
        }
        if (status_out) status_out[i] = st;
    }
    return total;
}

uint64_t wco_mv_num_keys(const wco_table *t) { return t->num_keys; }

/* retrieve_all_keys (multi_value_hash_table.cuh:561-598, gpu_engine.cuh:51-93):
 * a slot's key is output when that slot is the key's first entry along its
 * probe sequence (the lowest lane of the first window that holds it).
 * Output in slot order. */
uint64_t wco_mv_unique_keys(const wco_table *t, void *keys_out)
{
    uint64_t n = 0;
    for (uint64_t gid = 0; gid < t->capacity; gid++) {
        const uint64_t key = t->keys[gid];
        if (!valid_key(t, key)) continue;
        probe_t p;
        probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg, t->capacity, key, t->seed,
                    t->capacity);
        uint64_t guard = t->capacity / t->cg + 1;
        do {
            int64_t leader = -1;
            for (uint64_t r = 0; r < t->cg && leader < 0; r++)
                if (t->keys[p.pos[r]] == key) leader = (int64_t)p.pos[r];
            if (leader >= 0) {
                if ((uint64_t)leader == gid) {
                    if (keys_out) store_elem(keys_out, t->key_bytes, n, key);
                    n++;
                }
                break;
            }
        } while (--guard && probe_next(&p));
    }
    return n;
}

/* ------------------------------------------------------------------------ */
/* BucketListHashTable (bucket_list_hash_table.cuh) over BucketListStore      */
/* (storage.cuh:651-1454): a single-value table maps each key to a handle of  */
/* a list of value buckets in a shared pool.  The first bucket holds          */
/* min_bucket_size values and no header; every later bucket starts with a    */
/* header {previous bucket, size} and grows by grow_factor (float, ceilf) up  */
/* to max_bucket_size.  Handles pack {state, bucket index, count, values in   */
/* the newest bucket} in index_bits / counter_bits / size_bits (+2 state).    */
/* ------------------------------------------------------------------------ */

enum { BL_UNINIT = 0, BL_INIT = 1, BL_BLOCKING = 2, BL_FULL = 3 };

struct wco_bl {
    wco_table *keys;               /* SVHT<K, handle> (values hold packed handles) */
    int value_bytes;
    uint64_t capacity;             /* pool elements */
    uint64_t ib, cb, sb;           /* bucket index, counter, bucket size bits */
    float grow;
    uint64_t min_bucket, max_bucket, max_values;
    uint64_t next_free;
    uint64_t *pool_val, *pool_prev, *pool_size;
};

static uint64_t bl_head(const wco_bl *b) { return (1ull << b->ib) - 1; }

static uint64_t bl_pack(const wco_bl *b, int state, uint64_t index, uint64_t count, uint64_t tail)
{
    return (uint64_t)state | (index << 2) | (count << (2 + b->ib)) | (tail << (2 + b->ib + b->cb));
}

static void bl_unpack(const wco_bl *b, uint64_t h, int *state, uint64_t *index, uint64_t *count,
                      uint64_t *tail)
{
    *state = (int)(h & 3);
    *index = (h >> 2) & ((1ull << b->ib) - 1);
    *count = (h >> (2 + b->ib)) & ((1ull << b->cb) - 1);
    *tail = (h >> (2 + b->ib + b->cb)) & ((1ull << b->sb) - 1);
}

/* BucketListHashTable(key_capacity, value_capacity, seed, grow_factor,
 * min_bucket_size, max_bucket_size, max_values_per_key) (:106-121) with
 * BucketListStore<Value, index_bits, counter_bits, size_bits>.  NULL when
 * the store's configuration check (storage.cuh:990-1014) fails. */
wco_bl *wco_bl_create(int key_bytes, int value_bytes, uint64_t key_capacity,
                      uint64_t value_capacity, uint64_t seed, float grow_factor,
                      uint64_t min_bucket_size, uint64_t max_bucket_size,
                      uint64_t max_values_per_key, uint64_t index_bits, uint64_t counter_bits,
                      uint64_t size_bits, uint64_t cg)
{
    if (index_bits + counter_bits + size_bits + 2 > 64) return NULL;
    wco_bl *b = (wco_bl *)calloc(1, sizeof(wco_bl));
    b->ib = index_bits; b->cb = counter_bits; b->sb = size_bits;
    const uint64_t max_bucket_ok = (1ull << size_bits) - 1;
    if (!(value_capacity < bl_head(b) && grow_factor >= 1.0f && min_bucket_size >= 1 &&
          max_bucket_size >= min_bucket_size && max_bucket_size <= max_bucket_ok)) {
        free(b);
        return NULL;
    }
    b->value_bytes = value_bytes;
    b->capacity = value_capacity;
    b->grow = grow_factor;
    b->min_bucket = min_bucket_size;
    b->max_bucket = max_bucket_size;
    const uint64_t max_count = (1ull << counter_bits) - 1;
    b->max_values = max_values_per_key < max_count ? max_values_per_key : max_count;
    b->keys = wco_table_create(WCO_SVHT, key_bytes, 8, key_capacity, seed, cg, WCO_PROBE_DOUBLE,
                               WCO_HASH_MURMUR, WCO_HASH_MURMUR, 0, ~0ull, ~0ull);
    b->pool_val = (uint64_t *)calloc(value_capacity ? value_capacity : 1, 8);
    b->pool_prev = (uint64_t *)calloc(value_capacity ? value_capacity : 1, 8);
    b->pool_size = (uint64_t *)calloc(value_capacity ? value_capacity : 1, 8);
    wco_bl_init(b, seed);
    return b;
}

void wco_bl_destroy(wco_bl *b)
{
    if (!b) return;
    wco_table_destroy(b->keys);
    free(b->pool_val);
    free(b->pool_prev);
    free(b->pool_size);
    free(b);
}

/* init (:160-176; storage.cuh:1068-1098): keys empty, every handle
 * uninitialized, pool headers {head, min_bucket_size}, next free 0 */
void wco_bl_init(wco_bl *b, uint64_t seed)
{
    wco_table_init(b->keys, seed);
    const uint64_t u = bl_pack(b, BL_UNINIT, bl_head(b), 0, 0);
    for (uint64_t i = 0; i < b->keys->capacity; i++) b->keys->values[i] = u;
    for (uint64_t i = 0; i < b->capacity; i++) {
        b->pool_prev[i] = bl_head(b);
        b->pool_size[i] = b->min_bucket;
        b->pool_val[i] = 0;
    }
    b->next_free = 0;
}

uint64_t wco_bl_key_capacity(const wco_bl *b) { return b->keys->capacity; }

/* append (storage.cuh:1108-1285), one call after another */
static uint32_t bl_append(wco_bl *b, uint64_t *handle, uint64_t value)
{
    int state;
    uint64_t index, count, tail;
    bl_unpack(b, *handle, &state, &index, &count, &tail);
    if (state == BL_UNINIT) {
        const uint64_t alloc = b->next_free;
        b->next_free += b->min_bucket;
        if (alloc + b->min_bucket <= b->capacity) {
            b->pool_val[alloc] = value;
            *handle = bl_pack(b, BL_INIT, alloc, 1, 1);
            return WCO_ST_NONE;
        }
        *handle = bl_pack(b, BL_FULL, bl_head(b), 0, 0);
        return WCO_ST_OUT_OF_MEMORY;
    }
    if (state == BL_FULL) return WCO_ST_OUT_OF_MEMORY;
    if (count == b->max_values) return WCO_ST_MAX_VALUES_REACHED;
    const uint64_t cur_size = count <= b->min_bucket ? b->min_bucket : b->pool_size[index];
    if (tail == cur_size) {
        float grown = ceilf((float)cur_size * b->grow);
        float cap = (float)b->max_bucket;
        const uint64_t new_size = (uint64_t)(cap < grown ? cap : grown);
        const uint64_t alloc = b->next_free;
        b->next_free += new_size + 1;
        if (alloc + new_size + 1 <= b->capacity) {
            b->pool_val[alloc + 1] = value;
            b->pool_prev[alloc] = index;
            b->pool_size[alloc] = new_size;
            *handle = bl_pack(b, BL_INIT, alloc, count + 1, 1);
            return WCO_ST_NONE;
        }
        *handle = bl_pack(b, BL_FULL, index, count, tail);
        return WCO_ST_OUT_OF_MEMORY;
    }
    const uint64_t j = count + 1 <= b->min_bucket ? tail : tail + 1;
    b->pool_val[index + j] = value;
    *handle = bl_pack(b, BL_INIT, index, count + 1, tail + 1);
    return WCO_ST_NONE;
}

/* bulk insert (:235-326): key through the single-value table's insert
 * (none / duplicate_key / probing_length_exceeded / invalid_key), then the
 * append unless the key already holds max_values_per_key values; the
 * status is the sum of both and append errors are joined.  Like the
 * reference kernel (:300-322), no status is written for a key that found
 * no slot (invalid key, probing length exceeded). */
void wco_bl_insert(wco_bl *b, const void *keys, const void *values, uint64_t n,
                   uint64_t probing_length, uint32_t *status_out)
{
    for (uint64_t i = 0; i < n; i++) {
        uint32_t st = WCO_ST_UNKNOWN_ERROR;
        const int64_t slot = insert_impl(b->keys, load_elem(keys, b->keys->key_bytes, i),
                                         probing_length, &st);
        if (slot >= 0) {
            uint64_t *h = &b->keys->values[slot];
            int state;
            uint64_t index, count, tail;
            bl_unpack(b, *h, &state, &index, &count, &tail);
            uint32_t ast;
            if (count >= b->max_values) ast = WCO_ST_MAX_VALUES_REACHED;
            else ast = bl_append(b, h, load_elem(values, b->value_bytes, i));
            if (ast) join(b->keys, ast);
            st |= ast;
            if (status_out) status_out[i] = st;
        }
    }
}

/* the single-value table's retrieve of the handle (single_value_hash_table.cuh:268-307) */
static uint32_t bl_find(wco_bl *b, uint64_t key, uint64_t pl, uint64_t *handle)
{
    wco_table *t = b->keys;
    if (!valid_key(t, key)) {
        join(t, WCO_ST_INVALID_KEY);
        return WCO_ST_INVALID_KEY;
    }
    probe_t p;
    probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg, t->capacity, key, t->seed, pl);
    uint64_t guard = t->capacity / t->cg + 1;
    do {
        int any_empty = 0;
        for (uint64_t r = 0; r < t->cg; r++) {
            if (t->keys[p.pos[r]] == key) {
                *handle = t->values[p.pos[r]];
                return WCO_ST_NONE;
            }
            any_empty |= t->keys[p.pos[r]] == t->empty;
        }
        if (any_empty) {
            join(t, WCO_ST_KEY_NOT_FOUND);
            return WCO_ST_KEY_NOT_FOUND;
        }
    } while (--guard && probe_next(&p));
    join(t, WCO_ST_PROBING_LENGTH_EXCEEDED);
    return WCO_ST_PROBING_LENGTH_EXCEEDED;
}

/* for_each over a list (storage.cuh:1292-1343): the newest bucket's values
 * first, then every older bucket from its first place; out[index] */
static void bl_walk(const wco_bl *b, uint64_t h, void *out, uint64_t room)
{
    int state;
    uint64_t index, count, tail;
    bl_unpack(b, h, &state, &index, &count, &tail);
    if (state != BL_INIT || index == bl_head(b)) return;
    uint64_t ptr = index;
    uint64_t off = count <= b->min_bucket ? 0 : 1;
    uint64_t g = 0;
    for (uint64_t l = 0; l < tail; l++, g++)
        if (out && g < room) store_elem(out, b->value_bytes, g, b->pool_val[ptr + l + off]);
    while (g < count) {
        ptr = b->pool_prev[ptr];
        const int last = g >= count - b->min_bucket;
        const uint64_t size = last ? b->min_bucket : b->pool_size[ptr];
        off = last ? 0 : 1;
        for (uint64_t l = 0; l < size && g < count; l++, g++)
            if (out && g < room) store_elem(out, b->value_bytes, g, b->pool_val[ptr + l + off]);
    }
}

/* bulk num_values (:762-789, gpu_engine.cuh:466-504): the handle's count */
uint64_t wco_bl_num_values(wco_bl *b, const void *keys, uint64_t n, uint64_t *counts_out,
                           uint64_t probing_length, uint32_t *status_out)
{
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t h = 0, num = 0;
        const uint32_t st = bl_find(b, load_elem(keys, b->keys->key_bytes, i), probing_length, &h);
        if (st == WCO_ST_NONE) {
            int state;
            uint64_t index, tail;
            bl_unpack(b, h, &state, &index, &num, &tail);
        }
        if (counts_out) counts_out[i] = num;
        total += num;
        if (status_out) status_out[i] = st;
    }
    return total;
}

/* bulk retrieve (:375-466, gpu_engine.cuh:305-346): counts, scan, then each
 * key's list at its begin offset; a count that differs from the first
 * pass's is invalid_phase_overlap.  values_out NULL is a dry run. */
uint64_t wco_bl_retrieve(wco_bl *b, const void *keys, uint64_t n, uint64_t *begin_out,
                         uint64_t *end_out, void *values_out, uint64_t probing_length,
                         uint32_t *status_out)
{
    const uint64_t total = wco_bl_num_values(b, keys, n, end_out, probing_length, NULL);
    if (!values_out) {
        for (uint64_t i = 0; i < n && status_out; i++) status_out[i] = WCO_ST_DRY_RUN;
        join(b->keys, WCO_ST_DRY_RUN);
        return total;
    }
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; i++) {
        begin_out[i] = s;
        s += end_out[i];
        end_out[i] = s;
    }
    for (uint64_t i = 0; i < n; i++) {
        uint64_t h = 0, num = 0;
        uint32_t st = bl_find(b, load_elem(keys, b->keys->key_bytes, i), probing_length, &h);
        if (st == WCO_ST_NONE) {
            int state;
            uint64_t index, tail;
            bl_unpack(b, h, &state, &index, &num, &tail);
            char *dst = (char *)values_out + begin_out[i] * (uint64_t)b->value_bytes;
            bl_walk(b, h, dst, end_out[i] - begin_out[i]);
        }
        if (num != end_out[i] - begin_out[i]) {
            join(b->keys, WCO_ST_INVALID_PHASE_OVERLAP);
            st |= WCO_ST_INVALID_PHASE_OVERLAP;
        }
        if (status_out) status_out[i] = st;
    }
    return total;
}

/* num_keys = the key table's size (:719-726); num_values = the sum of all
 * handle counts (:797-818); the pool's next free index (load factor,
 * storage.cuh:1369-1396) */
uint64_t wco_bl_num_keys(const wco_bl *b) { return wco_size(b->keys); }

uint64_t wco_bl_total_values(const wco_bl *b)
{
    uint64_t n = 0;
    for (uint64_t i = 0; i < b->keys->capacity; i++) {
        if (!valid_key(b->keys, b->keys->keys[i])) continue;
        int state;
        uint64_t index, count, tail;
        bl_unpack(b, b->keys->values[i], &state, &index, &count, &tail);
        n += count;
    }
    return n;
}

uint64_t wco_bl_next_free(const wco_bl *b) { return b->next_free; }

/* retrieve_all_keys (:574-605): every valid key of the key table */
uint64_t wco_bl_all_keys(const wco_bl *b, void *keys_out)
{
    uint64_t n = 0;
    for (uint64_t i = 0; i < b->keys->capacity; i++) {
        const uint64_t k = b->keys->keys[i];
        if (!valid_key(b->keys, k)) continue;
        if (keys_out) store_elem(keys_out, b->keys->key_bytes, n, k);
        n++;
    }
    return n;
}

uint32_t wco_bl_peek_status(const wco_bl *b) { return b->keys->status; }

uint32_t wco_bl_pop_status(wco_bl *b)
{
    const uint32_t s = b->keys->status;
    b->keys->status = 0;
    return s;
}

/* ------------------------------------------------------------------------ */
/* MultiBucketHashTable (multi_bucket_hash_table.cuh): every slot holds a key */
/* and a bucket of `bucket` values; a key's values fill its last bucket       */
/* before a new slot is claimed.  Buckets larger than the group size are not  */
/* restated (the reference's loop over them reads value[rank] for every      */
/* chunk, :270-274), so bucket <= cg.                                         */
/* ------------------------------------------------------------------------ */

struct wco_mb {
    int key_bytes, value_bytes, scheme, h1, h2;
    uint64_t capacity, cg, bucket, seed, empty, tomb, empty_value, max_values;
    uint64_t *keys;
    uint64_t *vals; /* capacity * bucket */
    uint64_t num_keys, num_occupied;
    uint32_t status;
};

wco_mb *wco_mb_create(int key_bytes, int value_bytes, uint64_t bucket, uint64_t min_capacity,
                      uint64_t seed, uint64_t cg, int scheme, int h1, int h2, uint64_t empty_key,
                      uint64_t tombstone_key, uint64_t empty_value, uint64_t max_values_per_key)
{
    if (bucket == 0 || bucket > cg) return NULL;
    wco_mb *t = (wco_mb *)calloc(1, sizeof(wco_mb));
    t->key_bytes = key_bytes;
    t->value_bytes = value_bytes;
    t->scheme = scheme; t->h1 = h1; t->h2 = h2;
    t->cg = cg;
    t->bucket = bucket;
    t->capacity = wco_valid_capacity(min_capacity, cg);
    t->empty = empty_key & kmask(key_bytes);
    t->tomb = tombstone_key & kmask(key_bytes);
    t->empty_value = empty_value & kmask(value_bytes);
    t->max_values = max_values_per_key;
    t->keys = (uint64_t *)malloc((t->capacity ? t->capacity : 1) * 8);
    t->vals = (uint64_t *)malloc((t->capacity ? t->capacity : 1) * bucket * 8);
    wco_mb_init(t, seed);
    return t;
}

void wco_mb_destroy(wco_mb *t)
{
    if (!t) return;
    free(t->keys);
    free(t->vals);
    free(t);
}

uint64_t wco_mb_capacity(const wco_mb *t) { return t->capacity; }

/* init (:253-271): keys := empty, every bucket value := empty value,
 * counters zero */
void wco_mb_init(wco_mb *t, uint64_t seed)
{
    t->seed = seed & kmask(t->key_bytes);
    for (uint64_t i = 0; i < t->capacity; i++) t->keys[i] = t->empty;
    for (uint64_t i = 0; i < t->capacity * t->bucket; i++) t->vals[i] = t->empty_value;
    t->num_keys = 0;
    t->num_occupied = 0;
    t->status = 0;
}

static int mb_valid_key(const wco_mb *t, uint64_t k) { return k != t->empty && k != t->tomb; }

/* insert_into_bucket (:262-330), one thread after another: lane 0 and the
 * lanes past the bucket count as full ("first bucket value always written
 * after key insert"), the others hold value[lane]; the count so far grows
 * by the full ones; the first empty lane takes the value. */
static int mb_insert_into_bucket(wco_mb *t, uint64_t slot, uint64_t value, uint64_t num_values,
                                 uint32_t *st)
{
    const uint64_t B = t->bucket;
    uint64_t *const b = t->vals + slot * B;
    uint64_t empties = 0;
    for (uint64_t r = 1; r < B; r++)
        if (b[r] == t->empty_value) empties |= 1ull << r;
    num_values += B - (uint64_t)__builtin_popcountll(empties);
    if (num_values >= t->max_values) {
        *st = WCO_ST_DUPLICATE_KEY | WCO_ST_MAX_VALUES_REACHED;
        t->status |= *st;
        return 1;
    }
    if (empties) {
        b[__builtin_ctzll(empties)] = value;
        *st = num_values > 0 ? WCO_ST_DUPLICATE_KEY : WCO_ST_NONE;
        return 1;
    }
    return 0;
}

/* insert (:343-517): along the probe sequence, note the last slot that
 * holds the key and count bucket_size per such slot; once the count
 * reaches max_values_per_key, only the last bucket can take the value.  In
 * the first window with an empty slot, fill the last bucket if it has room,
 * else claim the empty slot with the value in its bucket's first place. */
static uint32_t mb_insert_one(wco_mb *t, uint64_t key, uint64_t value, uint64_t probing_length)
{
    const uint64_t B = t->bucket;
    if (!mb_valid_key(t, key)) {
        t->status |= WCO_ST_INVALID_KEY;
        return WCO_ST_INVALID_KEY;
    }
    if (value == t->empty_value) {
        t->status |= WCO_ST_INVALID_VALUE;
        return WCO_ST_INVALID_VALUE;
    }
    probe_t p;
    probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg, t->capacity, key, t->seed,
                probing_length);
    uint64_t num = 0, guard = t->capacity / t->cg + 1;
    int64_t last = -1;
    uint32_t st;
    do {
        int64_t hit_last = -1;
        uint64_t hits = 0, empties = 0;
        for (uint64_t r = 0; r < t->cg; r++) {
            const uint64_t k = t->keys[p.pos[r]];
            if (k == key) { hits++; hit_last = (int64_t)r; }
            if (k == t->empty) empties |= 1ull << r;
        }
        if (hits) last = (int64_t)p.pos[hit_last];
        num += B * hits;
        if (num >= t->max_values) {
            if (B == 1) {
                st = WCO_ST_DUPLICATE_KEY | WCO_ST_MAX_VALUES_REACHED;
                t->status |= st;
                return st;
            }
            st = WCO_ST_UNKNOWN_ERROR;
            mb_insert_into_bucket(t, (uint64_t)last, value, num - B, &st);
            return st;
        }
        if (empties) {
            if (B > 1 && last >= 0 && mb_insert_into_bucket(t, (uint64_t)last, value, num - B, &st))
                return st;
            const uint64_t slot = p.pos[__builtin_ctzll(empties)];
            t->keys[slot] = key;
            t->vals[slot * B] = value;
            t->num_occupied++;
            if (num == 0) t->num_keys++;
            return num > 0 ? WCO_ST_DUPLICATE_KEY : WCO_ST_NONE;
        }
    } while (--guard && probe_next(&p));
    if (B > 1 && last >= 0 && mb_insert_into_bucket(t, (uint64_t)last, value, num - B, &st))
        return st;
    st = WCO_ST_PROBING_LENGTH_EXCEEDED | (num > 0 ? WCO_ST_DUPLICATE_KEY : 0);
    t->status |= st;
    return st;
}

void wco_mb_insert(wco_mb *t, const void *keys, const void *values, uint64_t n,
                   uint64_t probing_length, uint32_t *status_out)
{
    for (uint64_t i = 0; i < n; i++) {
        const uint32_t st = mb_insert_one(t, load_elem(keys, t->key_bytes, i),
                                          load_elem(values, t->value_bytes, i), probing_length);
        if (status_out) status_out[i] = st;
    }
}

/* for_each (:786-846): windows of the probe sequence (probing length capped
 * at the capacity); a hit slot's non-empty values get the indices
 * num + bucket * (hits before it in the window) + place; the count grows by
 * bucket per hit less the empty places of the window's last hit; stop at a
 * window with an empty key or once the count reaches max_values_per_key. */
static uint32_t mb_for_each(wco_mb *t, uint64_t key, uint64_t probing_length, void *out,
                            uint64_t room, uint64_t *num_out)
{
    const uint64_t B = t->bucket;
    if (!mb_valid_key(t, key)) {
        *num_out = 0;
        t->status |= WCO_ST_INVALID_KEY;
        return WCO_ST_INVALID_KEY;
    }
    probe_t p;
    const uint64_t pl = probing_length < t->capacity ? probing_length : t->capacity;
    probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg, t->capacity, key, t->seed, pl);
    uint64_t num = 0, guard = t->capacity / t->cg + 1;
    do {
        uint64_t h = 0, last_empty = 0;
        int any_empty = 0;
        for (uint64_t r = 0; r < t->cg; r++) {
            const uint64_t k = t->keys[p.pos[r]];
            if (k == key) {
                const uint64_t j = num + B * h;
                uint64_t e = 0;
                for (uint64_t b = 0; b < B; b++) {
                    const uint64_t v = t->vals[p.pos[r] * B + b];
                    if (v != t->empty_value) {
                        if (out && j + b < room) store_elem(out, t->value_bytes, j + b, v);
                    } else {
                        e++;
                    }
                }
                last_empty = e;
                h++;
            }
            any_empty |= k == t->empty;
        }
        num += B * h - last_empty;
        if (any_empty || num >= t->max_values) {
            *num_out = num;
            if (num == 0) {
                t->status |= WCO_ST_KEY_NOT_FOUND;
                return WCO_ST_KEY_NOT_FOUND;
            }
            return WCO_ST_NONE;
        }
    } while (--guard && probe_next(&p));
    *num_out = num;
    t->status |= WCO_ST_PROBING_LENGTH_EXCEEDED;
    return WCO_ST_PROBING_LENGTH_EXCEEDED;
}

/* bulk num_values (:1013-1039, gpu_engine.cuh:466-504) */
uint64_t wco_mb_num_values(wco_mb *t, const void *keys, uint64_t n, uint64_t *counts_out,
                           uint64_t probing_length, uint32_t *status_out)
{
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t num = 0;
        const uint32_t st = mb_for_each(t, load_elem(keys, t->key_bytes, i), probing_length,
                                        NULL, 0, &num);
        if (counts_out) counts_out[i] = num;
        total += num;
        if (status_out) status_out[i] = st;
    }
    return total;
}

/* bulk retrieve (:574-680): counts, inclusive scan into end offsets, begin
 * offsets one behind, then each key's values at its begin offset; with
 * values_out NULL a dry run (per-key counts in end_out, status dry_run).
 * The reference writes values without a bound; here index >= the key's
 * count is not written (the counts come from the same walk). */
uint64_t wco_mb_retrieve(wco_mb *t, const void *keys, uint64_t n, uint64_t *begin_out,
                         uint64_t *end_out, void *values_out, uint64_t probing_length,
                         uint32_t *status_out)
{
    const uint64_t total = wco_mb_num_values(t, keys, n, end_out, probing_length, NULL);
    if (!values_out) {
        for (uint64_t i = 0; i < n && status_out; i++) status_out[i] = WCO_ST_DRY_RUN;
        t->status |= WCO_ST_DRY_RUN;
        return total;
    }
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; i++) {
        begin_out[i] = s;
        s += end_out[i];
        end_out[i] = s;
    }
    for (uint64_t i = 0; i < n; i++) {
        uint64_t num = 0;
        char *dst = (char *)values_out + begin_out[i] * (uint64_t)t->value_bytes;
        const uint32_t st = mb_for_each(t, load_elem(keys, t->key_bytes, i), probing_length, dst,
                                        end_out[i] - begin_out[i], &num);
        if (status_out) status_out[i] = st;
    }
    return total;
}

uint64_t wco_mb_num_keys(const wco_mb *t) { return t->num_keys; }
uint64_t wco_mb_num_occupied(const wco_mb *t) { return t->num_occupied; }

/* size (:1060-1082, gpu_engine.cuh:419-464): non-empty values of slots
 * with a valid key */
uint64_t wco_mb_size(const wco_mb *t)
{
    uint64_t n = 0;
    for (uint64_t i = 0; i < t->capacity; i++) {
        if (!mb_valid_key(t, t->keys[i])) continue;
        for (uint64_t b = 0; b < t->bucket; b++) n += t->vals[i * t->bucket + b] != t->empty_value;
    }
    return n;
}

/* retrieve_all_keys (:742-777, gpu_engine.cuh:51-93): a slot's key is
 * output when that slot is the lowest lane of the first window holding
 * the key; slot order */
uint64_t wco_mb_unique_keys(const wco_mb *t, void *keys_out)
{
    uint64_t n = 0;
    for (uint64_t gid = 0; gid < t->capacity; gid++) {
        const uint64_t key = t->keys[gid];
        if (!mb_valid_key(t, key)) continue;
        probe_t p;
        probe_begin(&p, t->scheme, t->h1, t->h2, t->key_bytes, t->cg, t->capacity, key, t->seed,
                    t->capacity);
        uint64_t guard = t->capacity / t->cg + 1;
        do {
            int64_t leader = -1;
            for (uint64_t r = 0; r < t->cg && leader < 0; r++)
                if (t->keys[p.pos[r]] == key) leader = (int64_t)p.pos[r];
            if (leader >= 0) {
                if ((uint64_t)leader == gid) {
                    if (keys_out) store_elem(keys_out, t->key_bytes, n, key);
                    n++;
                }
                break;
            }
        } while (--guard && probe_next(&p));
    }
    return n;
}

uint32_t wco_mb_peek_status(const wco_mb *t) { return t->status; }

uint32_t wco_mb_pop_status(wco_mb *t)
{
    const uint32_t s = t->status;
    t->status = 0;
    return s;
}

/* ------------------------------------------------------------------------ */
/* Bloom filter (bloom_filter.cuh:78-93 sizes, :168-192 insert,
 * :216-237 retrieve, :342-408 fpr)                                          */
/* ------------------------------------------------------------------------ */

struct wco_bloom {
    int key_bytes, slot_bytes, hasher;
    uint64_t cg, num_bits, num_slots, num_blocks, k, seed;
    uint64_t *words;
};

wco_bloom *wco_bloom_create(int key_bytes, int slot_bytes, uint64_t cg,
                            int hasher, uint64_t num_bits, uint64_t k,
                            uint64_t seed)
{
    wco_bloom *b = (wco_bloom *)calloc(1, sizeof(wco_bloom));
    b->key_bytes = key_bytes;
    b->slot_bytes = slot_bytes;
    b->hasher = hasher;
    b->cg = cg;
    b->num_bits = num_bits;
    b->num_slots = (num_bits + slot_bytes * 8 - 1) / (slot_bytes * 8);
    b->num_blocks = (b->num_slots + cg - 1) / cg;
    b->k = k;
    b->seed = seed & kmask(key_bytes);
    b->words = (uint64_t *)calloc(b->num_slots ? b->num_slots : 1, 8);
    return b;
}

void wco_bloom_destroy(wco_bloom *b)
{
    if (!b) return;
    free(b->words);
    free(b);
}

/* per-lane slot index and bit pattern of one key */
static void bloom_pattern(const wco_bloom *b, uint64_t key, uint64_t *idx,
                          uint64_t *mask)
{
    const uint64_t km = kmask(b->key_bytes);
    const uint64_t slot_bits = (uint64_t)b->slot_bytes * 8;
    const uint64_t block_bits = slot_bits * b->cg;
    const uint64_t blk = wco_hash(b->hasher, b->key_bytes, (key + b->seed) & km)
                         % b->num_blocks;
    for (uint64_t r = 0; r < b->cg; r++) {
        idx[r] = (blk * b->cg + r) % b->num_slots;
        mask[r] = 0;
    }
    for (uint64_t i = 0; i < b->k; i++) {
        const uint64_t h =
            wco_hash(b->hasher, b->key_bytes, (key + b->seed + i) & km) %
            block_bits;
        mask[h / slot_bits] |= 1ull << (h % slot_bits);
    }
}

void wco_bloom_insert(wco_bloom *b, const void *keys, uint64_t n)
{
    uint64_t idx[32], mask[32];
    for (uint64_t i = 0; i < n; i++) {
        bloom_pattern(b, load_elem(keys, b->key_bytes, i), idx, mask);
        for (uint64_t r = 0; r < b->cg; r++) b->words[idx[r]] |= mask[r];
    }
}

void wco_bloom_retrieve(const wco_bloom *b, const void *keys, uint64_t n,
                        uint8_t *flags_out)
{
    uint64_t idx[32], mask[32];
    for (uint64_t i = 0; i < n; i++) {
        bloom_pattern(b, load_elem(keys, b->key_bytes, i), idx, mask);
        int all = 1;
        for (uint64_t r = 0; r < b->cg; r++)
            all &= (b->words[idx[r]] & mask[r]) == mask[r];
        flags_out[i] = (uint8_t)all;
    }
}

uint64_t wco_bloom_num_slots(const wco_bloom *b) { return b->num_slots; }
uint64_t wco_bloom_num_blocks(const wco_bloom *b) { return b->num_blocks; }

void wco_bloom_words(const wco_bloom *b, uint64_t *out)
{
    memcpy(out, b->words, b->num_slots * 8);
}

/* bloom_filter.cuh:371-408 binom / fpr_base, :342-354 fpr */
static double bloom_binom(uint64_t n, uint64_t k, double p)
{
    double res = 1.0;
    for (uint64_t i = n - k + 1; i <= n; ++i) res = res * (double)i;
    for (uint64_t i = 1; i <= k; ++i) res = res / (double)i;
    return res * pow(p, (double)k) * pow(1.0 - p, (double)(n - k));
}

static double bloom_fpr_base(uint64_t m, uint64_t n, uint64_t k)
{
    return pow(1.0 - pow(1.0 - 1.0 / (double)m, (double)(n * k)), (double)k);
}

double wco_bloom_fpr(const wco_bloom *b, uint64_t n)
{
    const uint64_t block_bits = (uint64_t)b->slot_bytes * 8 * b->cg;
    const double bl = (double)(b->num_bits / block_bits);
    double res = 0.0;
    const uint64_t upper = 5 * n / (b->num_bits / block_bits);
    for (uint64_t i = 0; i < upper; ++i)
        res += bloom_binom(n, i, 1.0 / bl) *
               bloom_fpr_base((uint64_t)((double)b->num_bits / bl), i, b->k);
    return res;
}

/* ------------------------------------------------------------------------ */
/* synthetic data                                                            */
/* ------------------------------------------------------------------------ */

uint64_t wco_splitmix64(uint64_t *state)
{
    uint64_t z = (*state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* distinct keys: a bijective mix of the index (fmix is invertible), skipping
 * the two sentinels; for 32-bit keys the index is taken mod 2^32 */
void wco_gen_unique_keys(int key_bytes, uint64_t n, uint64_t seed, void *out)
{
    const uint64_t km = kmask(key_bytes);
    uint64_t j = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t k;
        do {
            const uint64_t x = (j++ + seed * 0x9e3779b97f4a7c15ull) & km;
            k = key_bytes == 4 ? (uint64_t)fmix32((uint32_t)x) : fmix64(x);
        } while (k == 0 || k == km);
        store_elem(out, key_bytes, i, k);
    }
}

void wco_gen_uniform(int bytes, uint64_t n, uint64_t seed, void *out)
{
    uint64_t s = seed;
    for (uint64_t i = 0; i < n; i++) store_elem(out, bytes, i, wco_splitmix64(&s));
}

static double u01(uint64_t *s)
{
    return (double)(wco_splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
}

/* rejection sampler of random_distributions.cuh:285-310 */
void wco_gen_zipf_ranks(uint64_t n_in, double s, uint64_t n_out, uint64_t seed,
                        uint64_t *ranks_out)
{
    uint64_t st = seed;
    const double t = (pow((double)n_in, 1.0 - s) - s) / (1.0 - s);
    for (uint64_t i = 0; i < n_out; i++) {
        uint64_t k;
        double y, rat;
        do {
            const double p = u01(&st);
            const double inv_b = (p * t <= 1.0)
                ? p * t
                : pow((p * t) * (1.0 - s) + s, 1.0 / (1.0 - s));
            k = (uint64_t)(inv_b + 1.0);
            y = u01(&st);
            const double bnd = (k <= 1) ? 1.0 / t : pow(inv_b, -s) / t;
            rat = pow((double)k, -s) / (bnd * t);
        } while (y >= rat);
        if (k > n_in) k = n_in;
        ranks_out[i] = k; /* 1-based rank; key index is k-1 */
    }
}

/* Zipf draws with one splitmix64 stream per output (the counter-based form
 * of the sampler above, as the library's generator draws them): output i's
 * stream is seeded with mix(seed ^ (i * golden + c)); ranks are 1-based,
 * or in[rank - 1] when `in` is given. */
static uint64_t sm_mix(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

void wco_gen_zipf_streams(const void *in, uint64_t n_in, void *out, uint64_t n_out, int bytes,
                          double s, uint64_t seed)
{
    const double t = (pow((double)n_in, 1.0 - s) - s) / (1.0 - s);
    for (uint64_t i = 0; i < n_out; i++) {
        const uint64_t st = sm_mix(seed ^ (i * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull));
        uint64_t draw = 0, k = 1;
        for (;;) {
            const double p = (double)(sm_mix(st + (++draw) * 0x9e3779b97f4a7c15ull) >> 11) *
                             (1.0 / 9007199254740992.0);
            const double pt = p * t;
            const double inv_b = pt <= 1.0 ? pt : pow(pt * (1.0 - s) + s, 1.0 / (1.0 - s));
            k = (uint64_t)(inv_b + 1.0);
            const double y = (double)(sm_mix(st + (++draw) * 0x9e3779b97f4a7c15ull) >> 11) *
                             (1.0 / 9007199254740992.0);
            const double b = k <= 1 ? 1.0 / t : pow(inv_b, -s) / t;
            const double rat = pow((double)k, -s) / (b * t);
            if (y < rat || draw >= (1u << 20)) break;
        }
        if (k > n_in) k = n_in;
        if (k < 1) k = 1;
        store_elem(out, bytes, i, in ? load_elem(in, bytes, k - 1) : k);
    }
}

/* ------------------------------------------------------------------------ */
/* multi-threaded CPU port of the reference insert/retrieve                  */
/* ------------------------------------------------------------------------ */

struct wco_mt_table {
    int key_bytes, value_bytes;
    uint64_t capacity, cg, seed;
    void *slots; /* AoS {K key; V value;} like storage.cuh:165-187 */
};

wco_mt_table *wco_mt_create(int key_bytes, int value_bytes, uint64_t capacity,
                            uint64_t cg, uint64_t seed)
{
    wco_mt_table *t = (wco_mt_table *)calloc(1, sizeof(wco_mt_table));
    t->key_bytes = key_bytes;
    t->value_bytes = value_bytes;
    t->capacity = capacity;
    t->cg = cg;
    t->seed = seed & kmask(key_bytes);
    t->slots = aligned_alloc(64, ((capacity * 2 * key_bytes + 63) / 64) * 64);
    return t;
}

void wco_mt_destroy(wco_mt_table *t)
{
    if (!t) return;
    free(t->slots);
    free(t);
}

typedef struct {
    wco_mt_table *t;
    const void *keys;
    const void *values;
    void *values_out;
    uint8_t *found_out;
    uint64_t begin, end;
} mt_job;

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

static void *mt_clear_worker(void *arg)
{
    mt_job *j = (mt_job *)arg;
    const size_t sb = 2 * (size_t)j->t->key_bytes;
    memset((char *)j->t->slots + j->begin * sb, 0, (j->end - j->begin) * sb);
    return NULL;
}

/* the reference's insert_impl with the key CAS and the value store after it
 * (single_value_hash_table.cuh:743-823, :222-225), one key per thread step */
#define MT_WORKERS(K, SUFFIX)                                                  \
    typedef struct { K key; K value; } mt_pair_##SUFFIX;                       \
    static void *mt_insert_##SUFFIX(void *arg)                                 \
    {                                                                          \
        mt_job *j = (mt_job *)arg;                                             \
        wco_mt_table *t = j->t;                                                \
        mt_pair_##SUFFIX *s = (mt_pair_##SUFFIX *)t->slots;                    \
        const K *keys = (const K *)j->keys;                                    \
        const K *vals = (const K *)j->values;                                  \
        const uint64_t cap = t->capacity, cg = t->cg;                          \
        const uint64_t base_mod = cap / cg - 1;                                \
        for (uint64_t i = j->begin; i < j->end; i++) {                         \
            const K key = keys[i];                                             \
            const uint64_t h = (K)(MT_HASH(K, (K)(key + (K)t->seed)));         \
            uint64_t pos0 = (K)(h);                                            \
            const uint64_t step =                                              \
                ((uint64_t)MT_HASH(K, (K)(key + (K)t->seed + 1)) % base_mod + 1) \
                * cg;                                                          \
            uint64_t w = 0;                                                    \
            for (; w <= cap / cg; w++) {                                       \
                int done = 0;                                                  \
                for (uint64_t r = 0; r < cg && !done; r++) {                   \
                    const uint64_t p =                                         \
                        ((uint64_t)(K)(pos0 + r) % cap + w * step) % cap;      \
                    if (__atomic_load_n(&s[p].key, __ATOMIC_RELAXED) == key) { \
                        s[p].value = vals[i];                                  \
                        done = 1;                                              \
                    }                                                          \
                }                                                              \
                for (uint64_t r = 0; r < cg && !done; r++) {                   \
                    const uint64_t p =                                         \
                        ((uint64_t)(K)(pos0 + r) % cap + w * step) % cap;      \
                    K expect = 0;                                              \
                    if (__atomic_load_n(&s[p].key, __ATOMIC_RELAXED) != 0)     \
                        continue;                                              \
                    if (__atomic_compare_exchange_n(&s[p].key, &expect, key,   \
                            0, __ATOMIC_RELAXED, __ATOMIC_RELAXED) ||          \
                        expect == key) {                                       \
                        s[p].value = vals[i];                                  \
                        done = 1;                                              \
                    }                                                          \
                }                                                              \
                if (done) break;                                               \
            }                                                                  \
        }                                                                      \
        return NULL;                                                           \
    }                                                                          \
    static void *mt_retrieve_##SUFFIX(void *arg)                               \
    {                                                                          \
        mt_job *j = (mt_job *)arg;                                             \
        wco_mt_table *t = j->t;                                                \
        const mt_pair_##SUFFIX *s = (const mt_pair_##SUFFIX *)t->slots;        \
        const K *keys = (const K *)j->keys;                                    \
        K *out = (K *)j->values_out;                                           \
        const uint64_t cap = t->capacity, cg = t->cg;                          \
        const uint64_t base_mod = cap / cg - 1;                                \
        for (uint64_t i = j->begin; i < j->end; i++) {                         \
            const K key = keys[i];                                             \
            const uint64_t pos0 = (K)(MT_HASH(K, (K)(key + (K)t->seed)));     \
            const uint64_t step =                                              \
                ((uint64_t)MT_HASH(K, (K)(key + (K)t->seed + 1)) % base_mod + 1) \
                * cg;                                                          \
            uint8_t found = 0;                                                 \
            for (uint64_t w = 0; w <= cap / cg; w++) {                         \
                int hit = -1, empty = 0;                                       \
                uint64_t p = 0;                                                \
                for (uint64_t r = 0; r < cg; r++) {                            \
                    p = ((uint64_t)(K)(pos0 + r) % cap + w * step) % cap;      \
                    if (s[p].key == key) { hit = (int)r; break; }              \
                    empty |= s[p].key == 0;                                    \
                }                                                              \
                if (hit >= 0) { out[i] = s[p].value; found = 1; break; }       \
                if (empty) break;                                              \
            }                                                                  \
            if (j->found_out) j->found_out[i] = found;                         \
        }                                                                      \
        return NULL;                                                           \
    }

#define MT_HASH(K, x) (sizeof(K) == 4 ? (uint64_t)fmix32((uint32_t)(x)) : fmix64((uint64_t)(x)))
MT_WORKERS(uint32_t, u32)
MT_WORKERS(uint64_t, u64)
#undef MT_HASH

static double mt_run(void *(*fn)(void *), wco_mt_table *t, const void *keys,
                     const void *values, void *values_out, uint8_t *found_out,
                     uint64_t n, int threads)
{
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    mt_job jobs[256];
    const double t0 = now_s();
    for (int i = 0; i < threads; i++) {
        jobs[i].t = t;
        jobs[i].keys = keys;
        jobs[i].values = values;
        jobs[i].values_out = values_out;
        jobs[i].found_out = found_out;
        jobs[i].begin = n * (uint64_t)i / threads;
        jobs[i].end = n * (uint64_t)(i + 1) / threads;
        pthread_create(&th[i], NULL, fn, &jobs[i]);
    }
    for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
    return now_s() - t0;
}

void wco_mt_clear(wco_mt_table *t, int threads)
{
    mt_run(mt_clear_worker, t, NULL, NULL, NULL, NULL, t->capacity, threads);
}

double wco_mt_insert(wco_mt_table *t, const void *keys, const void *values,
                     uint64_t n, int threads)
{
    return mt_run(t->key_bytes == 4 ? mt_insert_u32 : mt_insert_u64, t, keys,
                  values, NULL, NULL, n, threads);
}

double wco_mt_retrieve(wco_mt_table *t, const void *keys, uint64_t n,
                       void *values_out, uint8_t *found_out, int threads)
{
    return mt_run(t->key_bytes == 4 ? mt_retrieve_u32 : mt_retrieve_u64, t,
                  keys, NULL, values_out, found_out, n, threads);
}
