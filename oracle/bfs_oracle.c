/*
 * CPU oracle: exact level-synchronous BFS over packed permutation words.
 *
 * TEST INFRASTRUCTURE ONLY.  It is loaded by tests/, by __graft_entry__.smoke()
 * and by bench.py's cpu_baseline / --impl reference legs, always as the checker
 * or the timed CPU baseline, never by the product library.
 *
 * What it restates (paths relative to the TryDotAtwo/MultiGPUBFS tree):
 *   - the level loop of GraphDefinition.exact_layers,
 *     multigpubfs/graph_definition.py:109-117 (seen/frontier sets, layer = new states);
 *   - the packed-word CPU search of scripts/cpu_small_bfs.py:30-80 (symbols of
 *     `bits` bits, symbol i at bit offset i*bits, generators applied to words);
 *   - the permutation action child[i] = parent[g[i]], graph_definition.py:70-75;
 *   - the lexicographic (Lehmer) rank used by the exact permutation bitmap,
 *     crates/mgbfs-runtime/src/permutation_bitmap.rs:29-45, written here as the
 *     plain O(n^2) inversion count.
 *
 * The visited set is either a Lehmer-rank bitmap (all symbols distinct) or an
 * open-addressing set of packed words.  Threads share the visited set through
 * atomic test-and-set; each thread appends its new states to a private list
 * and the lists are concatenated, so layer sizes are exact and independent of
 * thread count.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#define ORACLE_OK 0
#define ORACLE_BAD_ARGUMENT 1
#define ORACLE_NO_MEMORY 2
#define ORACLE_CAPACITY 3
#define ORACLE_LAYERS 4

static inline uint64_t symbol_at(uint64_t w, uint32_t i, uint32_t bits) {
    uint64_t mask = (bits == 64) ? ~0ull : ((1ull << bits) - 1);
    return (w >> (i * bits)) & mask;
}

static inline uint64_t apply_generator(uint64_t w, const uint32_t* g, uint32_t n, uint32_t bits) {
    uint64_t out = 0;
    for (uint32_t i = 0; i < n; i++) out |= symbol_at(w, g[i], bits) << (i * bits);
    return out;
}

/* Lexicographic rank of a permutation of n distinct symbols 0..n-1:
 * sum_i (#{j > i : s_j < s_i}) * (n-1-i)!. */
static inline uint64_t lehmer_rank(uint64_t w, uint32_t n, uint32_t bits, const uint64_t* fact) {
    uint64_t rank = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint64_t si = symbol_at(w, i, bits), smaller = 0;
        for (uint32_t j = i + 1; j < n; j++) smaller += symbol_at(w, j, bits) < si;
        rank += smaller * fact[n - 1 - i];
    }
    return rank;
}

static inline uint64_t mix64(uint64_t x) {
    x ^= x >> 31; x *= 0x7fb5d329728ea185ull;
    x ^= x >> 27; x *= 0x81dadef4bc2dd44dull;
    x ^= x >> 33;
    return x;
}

typedef struct { uint64_t* data; uint64_t size, cap; } vec64;

static int vec_push(vec64* v, uint64_t x) {
    if (v->size == v->cap) {
        uint64_t cap = v->cap ? v->cap * 2 : 4096;
        uint64_t* d = (uint64_t*)realloc(v->data, cap * sizeof(uint64_t));
        if (!d) return ORACLE_NO_MEMORY;
        v->data = d; v->cap = cap;
    }
    v->data[v->size++] = x;
    return ORACLE_OK;
}

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : x > y;
}

/* Returns 1 when the word was newly inserted. */
static inline int visit(uint64_t w, int use_bitmap, uint64_t* table, uint64_t mask,
                        uint32_t n, uint32_t bits, const uint64_t* fact, int* full) {
    if (use_bitmap) {
        uint64_t r = lehmer_rank(w, n, bits, fact);
        uint64_t bit = 1ull << (r & 63);
        uint64_t old = __atomic_fetch_or(&table[r >> 6], bit, __ATOMIC_RELAXED);
        return !(old & bit);
    }
    uint64_t slot = mix64(w) & mask;
    for (uint64_t probe = 0; probe <= mask; probe++) {
        uint64_t cur = __atomic_load_n(&table[slot], __ATOMIC_RELAXED);
        if (cur == w) return 0;
        if (cur == ~0ull) {
            uint64_t expected = ~0ull;
            if (__atomic_compare_exchange_n(&table[slot], &expected, w, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED))
                return 1;
            if (expected == w) return 0;
        }
        slot = (slot + 1) & mask;
    }
    *full = 1;
    return 0;
}

/*
 * n, bits        : degree and bits per symbol (n*bits <= 64)
 * gens           : ngens x n generator table, child[i] = parent[g[i]]
 * start          : packed start word
 * use_bitmap     : 1 = Lehmer bitmap over n! ranks (symbols must be 0..n-1 distinct)
 * max_states     : hash capacity bound (ignored for the bitmap)
 * threads        : OpenMP threads (0 = all)
 * layers         : out, per-depth layer sizes (max_layers entries)
 * last, last_cap : out, the sorted deepest layer (up to last_cap words), and
 * prev, prev_cap : the sorted layer before it
 */
int oracle_packed_bfs(uint32_t n, uint32_t bits, uint32_t ngens, const uint32_t* gens,
                      uint64_t start, int use_bitmap, uint64_t max_states, int threads,
                      uint64_t* layers, uint32_t max_layers, uint32_t* n_layers,
                      uint64_t* last, uint64_t last_cap, uint64_t* last_count,
                      uint64_t* prev, uint64_t prev_cap, uint64_t* prev_count) {
    if (!n || n * bits > 64 || !ngens || !gens || !layers || !n_layers) return ORACLE_BAD_ARGUMENT;
    if (use_bitmap && n > 20) return ORACLE_BAD_ARGUMENT;
    for (uint32_t k = 0; k < ngens * n; k++) if (gens[k] >= n) return ORACLE_BAD_ARGUMENT;
    if (threads > 0) omp_set_num_threads(threads);
    uint64_t fact[21];
    fact[0] = 1;
    for (uint32_t i = 1; i <= 20; i++) fact[i] = fact[i - 1] * i;

    uint64_t words, mask = 0;
    if (use_bitmap) {
        words = (fact[n] + 63) / 64;
    } else {
        uint64_t slots = 1024;
        while (slots < 2 * max_states) slots <<= 1;
        words = slots; mask = slots - 1;
    }
    uint64_t* table = (uint64_t*)malloc(words * sizeof(uint64_t));
    if (!table) return ORACLE_NO_MEMORY;
    memset(table, use_bitmap ? 0 : 0xff, words * sizeof(uint64_t));

    int full = 0, rc = ORACLE_OK;
    visit(start, use_bitmap, table, mask, n, bits, fact, &full);
    uint64_t* frontier = (uint64_t*)malloc(sizeof(uint64_t));
    uint64_t fsize = 1, visited = 1;
    uint64_t* previous = NULL;
    uint64_t psize = 0;
    frontier[0] = start;
    uint32_t depth = 0;
    int nt = omp_get_max_threads();
    vec64* local = (vec64*)calloc((size_t)nt, sizeof(vec64));
    if (!local) { free(table); free(frontier); return ORACLE_NO_MEMORY; }

    while (fsize) {
        if (depth >= max_layers) { rc = ORACLE_LAYERS; break; }
        layers[depth++] = fsize;
        int oom = 0;
        #pragma omp parallel
        {
            vec64* mine = &local[omp_get_thread_num()];
            mine->size = 0;
            #pragma omp for schedule(dynamic, 4096)
            for (uint64_t i = 0; i < fsize; i++) {
                uint64_t w = frontier[i];
                for (uint32_t g = 0; g < ngens; g++) {
                    uint64_t c = apply_generator(w, gens + (uint64_t)g * n, n, bits);
                    if (visit(c, use_bitmap, table, mask, n, bits, fact, &full))
                        if (vec_push(mine, c)) oom = 1;
                }
            }
        }
        if (oom) { rc = ORACLE_NO_MEMORY; break; }
        if (full) { rc = ORACLE_CAPACITY; break; }
        uint64_t next = 0;
        for (int t = 0; t < nt; t++) next += local[t].size;
        visited += next;
        if (!use_bitmap && visited > max_states) { rc = ORACLE_CAPACITY; break; }
        uint64_t* nf = (uint64_t*)malloc((next ? next : 1) * sizeof(uint64_t));
        if (!nf) { rc = ORACLE_NO_MEMORY; break; }
        uint64_t at = 0;
        for (int t = 0; t < nt; t++) {
            memcpy(nf + at, local[t].data, local[t].size * sizeof(uint64_t));
            at += local[t].size;
        }
        if (next) {
            free(previous);
            previous = frontier; psize = fsize;
            frontier = nf; fsize = next;
        } else {
            free(nf);
            break;
        }
    }
    *n_layers = depth;
    if (rc == ORACLE_OK) {
        qsort(frontier, fsize, sizeof(uint64_t), cmp_u64);
        if (last_count) *last_count = fsize;
        if (last) memcpy(last, frontier, (fsize < last_cap ? fsize : last_cap) * sizeof(uint64_t));
        if (previous) qsort(previous, psize, sizeof(uint64_t), cmp_u64);
        if (prev_count) *prev_count = previous ? psize : 0;
        if (prev && previous) memcpy(prev, previous, (psize < prev_cap ? psize : prev_cap) * sizeof(uint64_t));
    }
    for (int t = 0; t < nt; t++) free(local[t].data);
    free(local); free(table); free(frontier); free(previous);
    return rc;
}

/* Lehmer rank of packed words, for rank known-answer tests. */
int oracle_lehmer_rank(uint32_t n, uint32_t bits, const uint64_t* words, uint64_t count, uint64_t* ranks) {
    if (!n || n > 20 || n * bits > 64) return ORACLE_BAD_ARGUMENT;
    uint64_t fact[21];
    fact[0] = 1;
    for (uint32_t i = 1; i <= 20; i++) fact[i] = fact[i - 1] * i;
    for (uint64_t i = 0; i < count; i++) ranks[i] = lehmer_rank(words[i], n, bits, fact);
    return ORACLE_OK;
}
