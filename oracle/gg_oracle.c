/*
 * gg_oracle.c -- CPU oracle for the all-pairs BFS (TEST INFRASTRUCTURE ONLY).
 *
 * This file is the checker, not the product: only tests/, the smoke() entry
 * and the cpu_baseline leg of bench.py may load it.  The CUDA engine never
 * links or calls it.
 *
 * It restates the queue BFS of the reference CPU calculator,
 * cppcode/cpuASPLqueue.cpp:54-96 (and its 2-D / 3-D twins
 * cppcode/cpuASPLpiece.cpp:180-231, cppcode/cpuASPLbox.cpp:111-165):
 *   - one BFS per representative source, two FIFO levels, a visited bitset of
 *     64-bit words (cpuASPLqueue.cpp:66-74);
 *   - every popped vertex adds `step` to the total (cpuASPLqueue.cpp:79);
 *   - the eccentricity of a source is the last level whose successor level is
 *     empty (cpuASPLqueue.cpp:86);
 *   - a source is "connected" when it popped all N vertices (cpuASPLqueue.cpp:90).
 * Unlike the reference it does not fold everything into a double: it returns
 * the exact per-level pair counts, per-source eccentricity and per-source
 * reach, from which every reference return convention (sentinels, N/M scaling,
 * level caps) is recomputed exactly by the Python side (oracle/oracle.py).
 *
 * The adjacency is CSR (row_ptr[n+1], col[]), built by oracle.py from the
 * lifted descriptions exactly as cpuASPLqueue.cpp:57-62 does.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

/* One BFS from `s`.  cnt_lvl[L] += number of vertices at distance L.
 * Returns the eccentricity (last non-empty level); *reached = vertices popped. */
static int bfs_one(int n, const int32_t *row_ptr, const int32_t *col, int s,
                   uint64_t *visited, int32_t *q_cur, int32_t *q_next,
                   uint64_t *cnt_lvl, int64_t *reached)
{
    memset(visited, 0, sizeof(uint64_t) * (size_t)((n >> 6) + 1));
    int n_cur = 0, n_next = 0, ecc = 0;
    int64_t popped = 0;
    visited[s >> 6] |= 1ULL << (s & 63);
    q_cur[n_cur++] = s;
    for (int step = 0; n_cur > 0; step++) {
        n_next = 0;
        for (int k = 0; k < n_cur; k++) {
            int v = q_cur[k];
            popped++;
            cnt_lvl[step]++;
            for (int e = row_ptr[v]; e < row_ptr[v + 1]; e++) {
                int to = col[e];
                uint64_t bit = 1ULL << (to & 63);
                if (visited[to >> 6] & bit) continue;
                visited[to >> 6] |= bit;
                q_next[n_next++] = to;
            }
        }
        if (n_next == 0) ecc = step;  /* cpuASPLqueue.cpp:86 */
        int32_t *t = q_cur; q_cur = q_next; q_next = t;
        n_cur = n_next;
    }
    *reached = popped;
    return ecc;
}

/* Work shared by the pthreads of one ggo_bfs call. */
typedef struct {
    int n; const int32_t *row_ptr, *col; int n_src; const int32_t *src;
    int32_t *ecc; int64_t *reached;
    int next;                 /* next source index to take */
    pthread_mutex_t mu;
    uint64_t *level_counts;   /* merged under mu */
    int failed;
} job_t;

static void *worker(void *arg)
{
    job_t *J = (job_t *)arg;
    int n = J->n;
    uint64_t *visited = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)((n >> 6) + 1));
    int32_t *q1 = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    int32_t *q2 = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    uint64_t *cnt = (uint64_t *)calloc((size_t)n, sizeof(uint64_t));
    if (!visited || !q1 || !q2 || !cnt) {
        pthread_mutex_lock(&J->mu); J->failed = 1; pthread_mutex_unlock(&J->mu);
    } else {
        for (;;) {
            pthread_mutex_lock(&J->mu);
            int i0 = J->next; J->next += 8;
            pthread_mutex_unlock(&J->mu);
            if (i0 >= J->n_src) break;
            int i1 = i0 + 8 < J->n_src ? i0 + 8 : J->n_src;
            for (int i = i0; i < i1; i++) {
                int64_t r = 0;
                int e = bfs_one(n, J->row_ptr, J->col, J->src[i], visited, q1, q2, cnt, &r);
                if (J->ecc) J->ecc[i] = e;
                if (J->reached) J->reached[i] = r;
            }
        }
        pthread_mutex_lock(&J->mu);
        for (int L = 0; L < n; L++) J->level_counts[L] += cnt[L];
        pthread_mutex_unlock(&J->mu);
    }
    free(visited); free(q1); free(q2); free(cnt);
    return NULL;
}

/*
 * All-pairs BFS from the listed sources.
 *   level_counts[n]  (zeroed here): level_counts[L] = #(source, vertex) pairs at distance L
 *   ecc[n_src]       (nullable):    eccentricity of each source within its component
 *   reached[n_src]   (nullable):    #vertices each source reaches (itself included)
 * n_threads <= 0 uses every online core.  Returns 0, or -1 on bad input / no memory.
 */
int ggo_bfs(int n, const int32_t *row_ptr, const int32_t *col,
            int n_src, const int32_t *src, int n_threads,
            uint64_t *level_counts, int32_t *ecc, int64_t *reached)
{
    if (n <= 0 || n_src < 0 || !row_ptr || !col || (n_src && !src) || !level_counts)
        return -1;
    for (int i = 0; i < n_src; i++)
        if (src[i] < 0 || src[i] >= n) return -1;
    for (int e = 0; e < row_ptr[n]; e++)
        if (col[e] < 0 || col[e] >= n) return -1;
    memset(level_counts, 0, sizeof(uint64_t) * (size_t)n);
    if (n_threads <= 0) n_threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 256) n_threads = 256;
    job_t J = {n, row_ptr, col, n_src, src, ecc, reached, 0, PTHREAD_MUTEX_INITIALIZER,
               level_counts, 0};
    pthread_t th[256];
    int started = 0;
    for (int t = 1; t < n_threads; t++)
        if (pthread_create(&th[started], NULL, worker, &J) == 0) started++;
    worker(&J);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    return J.failed ? -1 : 0;
}

/* Version tag so the test suite can tell which build it loaded. */
const char *ggo_version(void) { return "gg_oracle 1"; }
