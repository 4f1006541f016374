/* bfs_oracle.c -- CPU restatement of the reference's BFS path.
 *
 * TEST INFRASTRUCTURE ONLY (see bfs_oracle.h).  Plain C99, single threaded,
 * written for clarity rather than speed.  Compiled with -ffp-contract=off so
 * that the double arithmetic of the RMAT recursion is rounded step by step,
 * exactly like the device generator it checks.
 */
#include "bfs_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* el64 files                                                               */
/* ------------------------------------------------------------------------ */

/* Header rules of parse_edge_list_file_header (edge_list.cc:20-89) and the
 * checks of dist_edge_list::load_binary (dist_edge_list.cc:56-76): one text
 * line < 256 bytes ending in '\n', space separated long options, num_vertices
 * and num_edges > 0, --format el64, --is_deduped present. */
int or_el64_header(const char *path, int64_t *num_vertices, int64_t *num_edges,
                   int64_t *header_bytes)
{
    FILE *fp = fopen(path, "rb");
    if (!fp) { return -1; }
    char line[256];
    if (!fgets(line, sizeof line, fp)) { fclose(fp); return -2; }
    fclose(fp);
    size_t len = strlen(line);
    if (len == 0 || line[len - 1] != '\n') { return -2; }
    *header_bytes = (int64_t)len;
    line[len - 1] = '\0';
    int64_t nv = -1, ne = -1;
    int deduped = 0, el64 = 0;
    char *save = NULL;
    for (char *tok = strtok_r(line, " ", &save); tok; tok = strtok_r(NULL, " ", &save)) {
        if (!strcmp(tok, "--num_vertices") || !strcmp(tok, "--num_edges") ||
            !strcmp(tok, "--format")) {
            char *val = strtok_r(NULL, " ", &save);
            if (!val) { return -2; }
            if (!strcmp(tok, "--num_vertices")) { nv = atoll(val); }
            else if (!strcmp(tok, "--num_edges")) { ne = atoll(val); }
            else { el64 = !strcmp(val, "el64"); }
        } else if (!strcmp(tok, "--is_deduped")) {
            deduped = 1;
        } else if (!strcmp(tok, "--is_sorted") || !strcmp(tok, "--is_permuted") ||
                   !strcmp(tok, "--is_directed") || !strcmp(tok, "--is_undirected")) {
            /* accepted, no effect */
        } else {
            return -2; /* getopt_long would report an invalid field */
        }
    }
    if (nv <= 0 || ne <= 0) { return -3; }
    if (!el64) { return -4; }
    if (!deduped) { return -5; }
    *num_vertices = nv;
    *num_edges = ne;
    return 0;
}

int or_el64_load(const char *path, int64_t *src, int64_t *dst, int64_t num_edges)
{
    int64_t nv, ne, hb;
    int rc = or_el64_header(path, &nv, &ne, &hb);
    if (rc) { return rc; }
    if (ne != num_edges) { return -6; }
    FILE *fp = fopen(path, "rb");
    if (!fp) { return -1; }
    if (fseek(fp, (long)hb, SEEK_SET)) { fclose(fp); return -7; }
    int64_t pair[2];
    for (int64_t i = 0; i < ne; ++i) {
        if (fread(pair, sizeof pair, 1, fp) != 1) { fclose(fp); return -7; }
        src[i] = pair[0];
        dst[i] = pair[1];
    }
    fclose(fp);
    return 0;
}

/* Layout written by dump_bin (generator/edge_list_utils.h:170-197). */
int or_el64_write(const char *path, int64_t num_vertices, int64_t num_edges,
                  const int64_t *src, const int64_t *dst)
{
    FILE *fp = fopen(path, "wb");
    if (!fp) { return -1; }
    fprintf(fp, " --format el64 --num_edges %lld --num_vertices %lld"
                " --is_undirected --is_deduped --is_permuted\n",
            (long long)num_edges, (long long)num_vertices);
    for (int64_t i = 0; i < num_edges; ++i) {
        int64_t pair[2] = {src[i], dst[i]};
        if (fwrite(pair, sizeof pair, 1, fp) != 1) { fclose(fp); return -7; }
    }
    fclose(fp);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Graph construction                                                        */
/* ------------------------------------------------------------------------ */

/* graph_base.h:356-366 counts both endpoints of every edge, :404-415 carves
 * one block per vertex, :423-427 inserts (src->dst) then (dst->src) for each
 * edge in list order.  With one worker that order is the file order. */
int or_csr_build(int64_t n, int64_t m, const int64_t *src, const int64_t *dst,
                 int64_t *offsets, uint32_t *adj)
{
    for (int64_t v = 0; v <= n; ++v) { offsets[v] = 0; }
    for (int64_t i = 0; i < m; ++i) {
        if (src[i] < 0 || src[i] >= n || dst[i] < 0 || dst[i] >= n) { return -1; }
        offsets[src[i] + 1] += 1;
        offsets[dst[i] + 1] += 1;
    }
    for (int64_t v = 0; v < n; ++v) { offsets[v + 1] += offsets[v]; }
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    if (!fill) { return -2; }
    memcpy(fill, offsets, sizeof(int64_t) * (size_t)n);
    for (int64_t i = 0; i < m; ++i) {
        adj[fill[src[i]]++] = (uint32_t)dst[i];
        adj[fill[dst[i]]++] = (uint32_t)src[i];
    }
    free(fill);
    return 0;
}

static int has_arc(const int64_t *offsets, const uint32_t *adj, int64_t u, int64_t v)
{
    for (int64_t e = offsets[u]; e < offsets[u + 1]; ++e) {
        if ((int64_t)adj[e] == v) { return 1; }
    }
    return 0;
}

/* graph_base.h:110-134.  The duplicate test there looks only at adjacent
 * entries (std::adjacent_find), which is what is restated here. */
int or_graph_check(int64_t n, int64_t m, const int64_t *src, const int64_t *dst,
                   const int64_t *offsets, const uint32_t *adj)
{
    int ok = 1;
    for (int64_t i = 0; i < m; ++i) {
        if (!has_arc(offsets, adj, src[i], dst[i])) { ok = 0; }
        if (!has_arc(offsets, adj, dst[i], src[i])) { ok = 0; }
    }
    for (int64_t v = 0; v < n; ++v) {
        for (int64_t e = offsets[v] + 1; e < offsets[v + 1]; ++e) {
            if (adj[e] == adj[e - 1]) { ok = 0; }
        }
    }
    return ok;
}

/* ------------------------------------------------------------------------ */
/* Root picker                                                               */
/* ------------------------------------------------------------------------ */

/* lcg.h:11-27: 64-bit LCG, multiplier 6364136223846793005, increment 1, with
 * a jump-ahead constructor; hybrid_bfs_main.cc:136-144 draws rng() % n until
 * the vertex has nonzero degree. */
void or_pick_roots(int64_t n, const int64_t *offsets, uint64_t seed, int64_t k,
                   int64_t *roots)
{
    const uint64_t mul = 6364136223846793005ULL;
    uint64_t mul_k = mul, add_k = 1, ran = 1;
    for (uint64_t un = seed; un; un >>= 1) {
        if (un & 1) { ran = mul_k * ran + add_k; }
        add_k *= (mul_k + 1);
        mul_k *= mul_k;
    }
    uint64_t state = ran;
    for (int64_t s = 0; s < k; ++s) {
        int64_t v;
        do {
            state = mul * state + 1;
            /* the reference computes rng() % num_vertices() with a long
             * right operand: unsigned long % long -> unsigned modulo */
            v = (int64_t)(state % (uint64_t)n);
        } while (offsets[v + 1] - offsets[v] == 0);
        roots[s] = v;
    }
}

/* ------------------------------------------------------------------------ */
/* BFS oracles                                                               */
/* ------------------------------------------------------------------------ */

/* hybrid_bfs.cc:285-307: serial FIFO BFS over out_neighbors. */
void or_bfs_depth(int64_t n, const int64_t *offsets, const uint32_t *adj,
                  int64_t source, int32_t *depth)
{
    for (int64_t v = 0; v < n; ++v) { depth[v] = -1; }
    int64_t *q = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    if (!q) { return; }
    int64_t head = 0, tail = 0;
    q[tail++] = source;
    depth[source] = 0;
    while (head < tail) {
        int64_t u = q[head++];
        for (int64_t e = offsets[u]; e < offsets[u + 1]; ++e) {
            int64_t v = adj[e];
            if (depth[v] == -1) {
                depth[v] = depth[u] + 1;
                q[tail++] = v;
            }
        }
    }
    free(q);
}

/* hybrid_bfs.cc:281-379.  Returns the vertex u at which the reference's
 * ascending loop stops (the u its LOG lines name), or -1 when the check
 * passes. */
int64_t or_check_first_bad(int64_t n, const int64_t *offsets, const uint32_t *adj,
                           int64_t source, const int64_t *parent, int32_t *depth)
{
    or_bfs_depth(n, offsets, adj, source, depth);
    for (int64_t u = 0; u < n; ++u) {
        if (depth[u] >= 0 && parent[u] >= 0) {
            if (u == source) {
                if (!(parent[u] == u && depth[u] == 0)) { return u; }
                continue;
            }
            int found = 0;
            for (int64_t e = offsets[u]; e < offsets[u + 1]; ++e) {
                int64_t v = adj[e];
                if (v == parent[u]) {
                    /* "Wrong depths" breaks out with found still 0 */
                    if (depth[v] == depth[u] - 1) { found = 1; }
                    break;
                }
            }
            if (!found) { return u; }
        } else if ((depth[u] < 0) != (parent[u] < 0)) {
            return u;
        }
    }
    return -1;
}

/* hybrid_bfs::check's verdict: 1 = pass. */
int or_check(int64_t n, const int64_t *offsets, const uint32_t *adj,
             int64_t source, const int64_t *parent, int32_t *depth)
{
    return or_check_first_bad(n, offsets, adj, source, parent, depth) < 0;
}

void or_min_parent(int64_t n, const int64_t *offsets, const uint32_t *adj,
                   int64_t source, const int32_t *depth, int64_t *parent)
{
    for (int64_t v = 0; v < n; ++v) {
        int64_t deg = offsets[v + 1] - offsets[v];
        if (depth[v] < 0) {
            parent[v] = deg != 0 ? -deg : -1;
        } else if (v == source) {
            parent[v] = v;
        } else {
            int64_t best = -1;
            for (int64_t e = offsets[v]; e < offsets[v + 1]; ++e) {
                int64_t u = adj[e];
                if (depth[u] == depth[v] - 1 && (best < 0 || u < best)) { best = u; }
            }
            parent[v] = best;
        }
    }
}

/* hybrid_bfs.cc:401-414: sum of degrees of reached vertices, halved. */
int64_t or_count_traversed(int64_t n, const int64_t *offsets, const int64_t *parent)
{
    int64_t sum = 0;
    for (int64_t v = 0; v < n; ++v) {
        if (parent[v] >= 0) { sum += offsets[v + 1] - offsets[v]; }
    }
    return sum / 2;
}

/* ---- connected components ------------------------------------------------ */

/* components::run (components.cc:38-118) as its serial elision executes
 * it.  Every vertex starts as its own component; a pass visits every arc
 * (src, dst) and lowers component[src] to component[dst] when that is
 * smaller; then each vertex's label is replaced by its label's label until
 * it is a fixed point (pointer jumping); passes repeat until one changes
 * nothing.  The worklist pushes each vertex at its head (worklist.h
 * append), so a pass visits vertices in descending order; pointer jumping
 * runs in ascending order.  Returns the number of passes (the last, which
 * changed nothing, included) -- the `num_iters` the reference prints. */
int64_t or_components(int64_t n, const int64_t *offsets, const uint32_t *adj,
                      int64_t *component, int64_t *size, int64_t *num_components)
{
    for (int64_t v = 0; v < n; ++v) {
        component[v] = v;
        size[v] = 0;
    }
    int64_t iters;
    for (iters = 1;; ++iters) {
        int changed = 0;
        for (int64_t s = n - 1; s >= 0; --s) {
            for (int64_t e = offsets[s]; e < offsets[s + 1]; ++e) {
                int64_t d = adj[e];
                if (component[d] < component[s]) {
                    component[s] = component[d];
                    changed = 1;
                }
            }
        }
        if (!changed) { break; }
        for (int64_t v = 0; v < n; ++v) {
            while (component[v] != component[component[v]]) {
                component[v] = component[component[v]];
            }
        }
    }
    int64_t count = 0;
    for (int64_t v = 0; v < n; ++v) { size[component[v]] += 1; }
    for (int64_t v = 0; v < n; ++v) { count += size[v] > 0; }
    *num_components = count;
    return iters;
}

typedef struct {
    int64_t label, vertex;
} or_label_pair;

static int or_label_cmp(const void *a, const void *b)
{
    const or_label_pair *x = a, *y = b;
    if (x->label != y->label) { return x->label < y->label ? -1 : 1; }
    return x->vertex < y->vertex ? -1 : (x->vertex > y->vertex);
}

/* components::check (components.cc:155-200): for each distinct label, a
 * serial BFS from the last vertex carrying it (the label_to_source map is
 * filled in ascending vertex order) must meet only that label, and every
 * vertex must be visited by one of these searches.  Returns 1 = PASS. */
int or_components_check(int64_t n, const int64_t *offsets, const uint32_t *adj,
                        const int64_t *component)
{
    or_label_pair *pairs = malloc(sizeof(*pairs) * (n ? n : 1));
    char *visited = calloc(n ? n : 1, 1);
    int64_t *q = malloc(sizeof(int64_t) * (n ? n : 1));
    for (int64_t v = 0; v < n; ++v) {
        pairs[v].label = component[v];
        pairs[v].vertex = v;
    }
    qsort(pairs, n, sizeof(*pairs), or_label_cmp);
    int ok = 1;
    for (int64_t i = 0; i < n && ok; ++i) {
        if (i + 1 < n && pairs[i + 1].label == pairs[i].label) { continue; }
        const int64_t label = pairs[i].label, source = pairs[i].vertex;
        visited[source] = 1;
        int64_t head = 0, tail = 0;
        q[tail++] = source;
        while (head < tail && ok) {
            const int64_t u = q[head++];
            for (int64_t e = offsets[u]; e < offsets[u + 1]; ++e) {
                const int64_t v = adj[e];
                if (component[v] != label) {
                    ok = 0;
                    break;
                }
                if (!visited[v]) {
                    visited[v] = 1;
                    q[tail++] = v;
                }
            }
        }
    }
    for (int64_t v = 0; v < n && ok; ++v) {
        if (!visited[v]) { ok = 0; }
    }
    free(pairs);
    free(visited);
    free(q);
    return ok;
}

/* run_beamer's control flow (hybrid_bfs.cc:152-191) over a level profile.
 * Both step kinds discover exactly the next BFS level, so the per-level
 * vertex counts and degree sums fix every decision:
 *   - scout after a top-down step = sum of degrees of the new vertices
 *     (recovered from the -deg parent encoding, :93 and :438);
 *   - awake after a bottom-up step = number of new vertices (:139-142);
 *   - edges_to_check starts at 2m and shrinks only on top-down steps;
 *   - scout is reset to 1 after a bottom-up phase (:180). */
int or_beamer_sequence(int64_t n, int64_t m, const int64_t *offsets,
                       const int32_t *depth, int64_t source, int64_t alpha,
                       int64_t beta, char *dirs, int64_t *found, int max_steps)
{
    int32_t maxd = 0;
    for (int64_t v = 0; v < n; ++v) { if (depth[v] > maxd) { maxd = depth[v]; } }
    int64_t levels = (int64_t)maxd + 2; /* one empty level past the last */
    int64_t *cnt = (int64_t *)calloc((size_t)levels, sizeof(int64_t));
    int64_t *deg = (int64_t *)calloc((size_t)levels, sizeof(int64_t));
    if (!cnt || !deg) { free(cnt); free(deg); return -1; }
    for (int64_t v = 0; v < n; ++v) {
        if (depth[v] >= 0) {
            cnt[depth[v]] += 1;
            deg[depth[v]] += offsets[v + 1] - offsets[v];
        }
    }
    int steps = 0;
    int64_t f = 0; /* level of the current frontier */
    int64_t edges_to_check = 2 * m;
    int64_t scout = offsets[source + 1] - offsets[source];
    while (f < levels && cnt[f] > 0) {
        if (scout > edges_to_check / alpha) {
            int64_t awake = cnt[f], old;
            do {
                old = awake;
                awake = (f + 1 < levels) ? cnt[f + 1] : 0;
                if (steps >= max_steps) { free(cnt); free(deg); return -1; }
                dirs[steps] = 'B';
                found[steps] = awake;
                ++steps;
                ++f;
            } while (awake >= old || awake > n / beta);
            scout = 1;
        } else {
            edges_to_check -= scout;
            scout = (f + 1 < levels) ? deg[f + 1] : 0;
            if (steps >= max_steps) { free(cnt); free(deg); return -1; }
            dirs[steps] = 'T';
            found[steps] = (f + 1 < levels) ? cnt[f + 1] : 0;
            ++steps;
            ++f;
        }
    }
    if (steps < max_steps) { dirs[steps] = '\0'; }
    free(cnt);
    free(deg);
    return steps;
}

/* Serial run_beamer / top-down-only / bottom-up-only. */
int or_run_bfs(int64_t n, int64_t m, const int64_t *offsets, const uint32_t *adj,
               int64_t source, int64_t alpha, int64_t beta, int mode,
               int64_t *parent, int32_t *depth, char *dirs, int max_steps)
{
    /* clear() (hybrid_bfs.cc:433-443) */
    for (int64_t v = 0; v < n; ++v) {
        int64_t d = offsets[v + 1] - offsets[v];
        parent[v] = d != 0 ? -d : -1;
        depth[v] = -1;
    }
    int64_t *queue = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t *new_parent = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
    if (!queue || !new_parent) { free(queue); free(new_parent); return -1; }
    for (int64_t v = 0; v < n; ++v) { new_parent[v] = -1; }
    int64_t qs = 0, qe = 0; /* current window [qs, qe) */
    queue[qe++] = source;
    parent[source] = source;
    depth[source] = 0;
    int32_t level = 0;
    int steps = 0;
    int64_t edges_to_check = 2 * m;
    int64_t scout = offsets[source + 1] - offsets[source];
    int in_bottom_up = 0;
    int64_t awake = 0, old_awake = 0;

    while (qe > qs) {
        int bottom_up;
        if (mode == 1) { bottom_up = 0; }
        else if (mode == 2) { bottom_up = 1; }
        else if (in_bottom_up) { bottom_up = 1; }
        else if (scout > edges_to_check / alpha) {
            bottom_up = 1;
            in_bottom_up = 1;
            awake = qe - qs;
        } else { bottom_up = 0; }

        int64_t next = qe;
        if (!bottom_up) {
            if (mode == 0) { edges_to_check -= scout; }
            scout = 0;
            for (int64_t i = qs; i < qe; ++i) {
                int64_t u = queue[i];
                for (int64_t e = offsets[u]; e < offsets[u + 1]; ++e) {
                    int64_t v = adj[e];
                    int64_t cur = parent[v];
                    if (cur < 0) {
                        parent[v] = u;
                        depth[v] = level + 1;
                        queue[next++] = v;
                        scout += -cur;
                    }
                }
            }
        } else {
            old_awake = awake;
            /* pass 1: parent_ frozen, discoveries go to new_parent */
            for (int64_t c = 0; c < n; ++c) {
                if (parent[c] >= 0) { continue; }
                int64_t b = offsets[c], e = offsets[c + 1];
                /* find.h:14-44: single steps until the rest is a multiple of
                 * four, then each group of four in reverse order */
                int64_t hit = -1;
                while ((e - b) % 4 != 0) {
                    int64_t p = adj[b++];
                    if (parent[p] >= 0) { hit = p; break; }
                }
                while (hit < 0 && b != e) {
                    int64_t e4 = adj[b], e3 = adj[b + 1], e2 = adj[b + 2], e1 = adj[b + 3];
                    b += 4;
                    if (parent[e1] >= 0) { hit = e1; }
                    else if (parent[e2] >= 0) { hit = e2; }
                    else if (parent[e3] >= 0) { hit = e3; }
                    else if (parent[e4] >= 0) { hit = e4; }
                }
                if (hit >= 0) { new_parent[c] = hit; }
            }
            /* pass 2: commit */
            awake = 0;
            for (int64_t v = 0; v < n; ++v) {
                if (parent[v] < 0 && new_parent[v] >= 0) {
                    parent[v] = new_parent[v];
                    depth[v] = level + 1;
                    queue[next++] = v;
                    awake += 1;
                }
            }
        }
        if (steps < max_steps) { dirs[steps] = bottom_up ? 'B' : 'T'; }
        ++steps;
        qs = qe;
        qe = next;
        level += 1;
        if (mode == 0 && bottom_up) {
            if (!(awake >= old_awake || awake > n / beta)) {
                in_bottom_up = 0;
                scout = 1;
            }
        }
    }
    if (steps < max_steps) { dirs[steps] = '\0'; }
    free(queue);
    free(new_parent);
    return steps;
}

/* ------------------------------------------------------------------------ */
/* Seeded RMAT generator                                                      */
/* ------------------------------------------------------------------------ */

/* Philox4x32 with 10 rounds, as published by Salmon, Moraes, Dror and Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3" (SC'11): round multipliers
 * 0xD2511F53 / 0xCD9E8D57, key schedule increments 0x9E3779B9 / 0xBB67AE85. */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Draw j of attempt t of edge i: block j/2 of the counter (i, t), upper or
 * lower 64 bits, top 53 bits scaled into [0, 1). */
static double rmat_uniform(uint64_t seed, int64_t i, uint32_t t, uint32_t j)
{
    uint32_t ctr[4] = {(uint32_t)(uint64_t)i, (uint32_t)((uint64_t)i >> 32), t, j >> 1};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    or_philox4x32(ctr, key, out);
    uint64_t w = (j & 1) ? (((uint64_t)out[2] << 32) | out[3])
                         : (((uint64_t)out[0] << 32) | out[1]);
    return (double)(w >> 11) * (1.0 / 9007199254740992.0);
}

#define OR_MAX_ATTEMPTS 4096

/* rmat_generator.h:91-140, one attempt. */
static void rmat_attempt(int scale, double a, double b, double c, double d,
                         uint64_t seed, int64_t i, uint32_t t,
                         int64_t *src, int64_t *dst)
{
    double A = a, B = b, C = c, D = d;
    int64_t si = 0, sj = 0;
    int64_t bit = (int64_t)1 << (scale - 1);
    uint32_t j = 0;
    for (;;) {
        double r = rmat_uniform(seed, i, t, j++);
        if (r > A) {
            if (r <= A + B) { sj |= bit; }
            else if (r <= A + B + C) { si |= bit; }
            else { sj |= bit; si |= bit; }
        }
        if (bit == 1) { break; }
        A *= (9.5 + rmat_uniform(seed, i, t, j++)) / 10;
        B *= (9.5 + rmat_uniform(seed, i, t, j++)) / 10;
        C *= (9.5 + rmat_uniform(seed, i, t, j++)) / 10;
        D *= (9.5 + rmat_uniform(seed, i, t, j++)) / 10;
        {
            double norm = 1.0 / (A + B + C + D);
            A *= norm;
            B *= norm;
            C *= norm;
        }
        D = 1.0 - (A + B + C);
        bit >>= 1;
    }
    *src = si;
    *dst = sj;
}

void or_rmat_edges(int scale, int64_t num_edges, double a, double b, double c,
                   double d, uint64_t seed, int64_t *src, int64_t *dst)
{
    for (int64_t i = 0; i < num_edges; ++i) {
        uint32_t t = 0;
        do {
            rmat_attempt(scale, a, b, c, d, seed, i, t, &src[i], &dst[i]);
            ++t;
        } while (src[i] == dst[i] && t < OR_MAX_ATTEMPTS);
    }
}

/* ------------------------------------------------------------------------ */
/* The reference generator's own stream (rmat_generator.h, prng_engine.hpp)   */
/* ------------------------------------------------------------------------ */

/* sitmo::prng_engine (generator/prng_engine.hpp, MIT licence, vendored by the
 * reference): Threefish-256 as specified for Skein 1.3, cut to 20 rounds,
 * tweak zero, key (seed, 0, 0, 0), encrypting the counter (block, 0, 0, 0).
 * Words are mixed in pairs (x, y) -> (x + y, rotl(y, R) ^ (x + y)); even
 * rounds pair words 0-1 and 2-3, odd rounds 0-3 and 2-1 (the Threefish-256
 * permutation); subkey s = (k[s], k[s+1], k[s+2], k[s+3] + s) mod-5 indexed,
 * k[4] = C240 ^ k0 ^ k1 ^ k2 ^ k3, is added before every fourth round and
 * after the last (s = 5). */
void or_threefish20(uint64_t key0, uint64_t block, uint64_t out[4])
{
    static const int rot[8][2] = {{14, 16}, {52, 57}, {23, 40}, {5, 37},
                                  {25, 33}, {46, 12}, {58, 22}, {32, 32}};
    uint64_t k[5] = {key0, 0, 0, 0, 0};
    k[4] = 0x1BD11BDAA9FC1A22ull ^ k[0] ^ k[1] ^ k[2] ^ k[3];
    uint64_t x[4] = {block, 0, 0, 0};
    for (int r = 0; r <= 20; ++r) {
        if (r % 4 == 0) {
            int sub = r / 4;
            for (int w = 0; w < 4; ++w) { x[w] += k[(sub + w) % 5]; }
            x[3] += (uint64_t)sub;
        }
        if (r == 20) { break; }
        int a = 0, b = (r % 2 == 0) ? 1 : 3, c = 2, d = (r % 2 == 0) ? 3 : 1;
        int ra = rot[r % 8][0], rc = rot[r % 8][1];
        x[a] += x[b];
        x[b] = ((x[b] << ra) | (x[b] >> (64 - ra))) ^ x[a];
        x[c] += x[d];
        x[d] = ((x[d] << rc) | (x[d] >> (64 - rc))) ^ x[c];
    }
    for (int w = 0; w < 4; ++w) { out[w] = x[w]; }
}

/* 32-bit output t of the engine seeded with `seed`: half (low for even t,
 * high for odd t) of word (t % 8) / 2 of block t / 8. */
uint32_t or_sitmo_output(uint32_t seed, uint64_t t)
{
    uint64_t o[4];
    or_threefish20(seed, t >> 3, o);
    uint64_t w = o[(t & 7) >> 1];
    return (t & 1) ? (uint32_t)(w >> 32) : (uint32_t)w;
}

/* A sequential reader of the stream that keeps the current block. */
typedef struct {
    uint32_t seed;
    uint64_t t, block;
    uint64_t o[4];
    int have;
} or_sitmo;

static uint32_t sitmo_next(or_sitmo *g)
{
    uint64_t blk = g->t >> 3;
    if (!g->have || blk != g->block) {
        or_threefish20(g->seed, blk, g->o);
        g->block = blk;
        g->have = 1;
    }
    uint64_t w = g->o[(g->t & 7) >> 1];
    uint32_t u = (g->t & 1) ? (uint32_t)(w >> 32) : (uint32_t)w;
    g->t += 1;
    return u;
}

/* libstdc++'s generate_canonical<double, 53> over a 32-bit engine (two
 * outputs: (u0 + u1 * 2^32) / 2^64, one rounding at the sum; a result of 1
 * becomes nextafter(1, 0)), which uniform_real_distribution<double>(0, 1)
 * returns unchanged. */
static double sitmo_uniform(or_sitmo *g)
{
    double sum = 0.0, scale = 1.0;
    for (int k = 0; k < 2; ++k) {
        sum += (double)sitmo_next(g) * scale;
        scale *= 4294967296.0;
    }
    double r = sum / scale;
    return r >= 1.0 ? 1.0 - 1.0 / 9007199254740992.0 : r;
}

/* next_edge (rmat_generator.h:91-140) on the reference stream. */
static void sitmo_next_edge(int scale, double a, double b, double c, double d, or_sitmo *g,
                            int64_t *src, int64_t *dst)
{
    double A = a, B = b, C = c, D = d;
    int64_t si = 0, sj = 0;
    int64_t bit = (int64_t)1 << (scale - 1);
    for (;;) {
        double r = sitmo_uniform(g);
        if (r > A) {
            if (r <= A + B) { sj |= bit; }
            else if (r <= A + B + C) { si |= bit; }
            else { sj |= bit; si |= bit; }
        }
        if (bit == 1) { break; }
        A *= (9.5 + sitmo_uniform(g)) / 10;
        B *= (9.5 + sitmo_uniform(g)) / 10;
        C *= (9.5 + sitmo_uniform(g)) / 10;
        D *= (9.5 + sitmo_uniform(g)) / 10;
        {
            double norm = 1.0 / (A + B + C + D);
            A *= norm;
            B *= norm;
            C *= norm;
        }
        D = 1.0 - (A + B + C);
        bit >>= 1;
    }
    *src = si;
    *dst = sj;
}

/* rmat_fill (rmat_generator.h:145-193) run serially: edge after edge from
 * the start of the stream, then every self loop, in edge order, re-rolled
 * with further edges from where the stream stands.  Returns 0, or -1 when
 * a degenerate A-D keeps producing self loops. */
int or_rmat_stream_edges(int scale, int64_t num_edges, double a, double b, double c,
                         double d, uint32_t seed, int64_t *src, int64_t *dst)
{
    or_sitmo g = {seed, 0, 0, {0, 0, 0, 0}, 0};
    for (int64_t i = 0; i < num_edges; ++i) {
        sitmo_next_edge(scale, a, b, c, d, &g, &src[i], &dst[i]);
    }
    int64_t draws = 0;
    for (int64_t i = 0; i < num_edges; ++i) {
        while (src[i] == dst[i]) {
            if (++draws > (int64_t)OR_MAX_ATTEMPTS * (num_edges + 1)) { return -1; }
            sitmo_next_edge(scale, a, b, c, d, &g, &src[i], &dst[i]);
        }
    }
    return 0;
}

typedef struct { uint64_t key; uint64_t idx; } or_keyed;

static int cmp_keyed(const void *pa, const void *pb)
{
    const or_keyed *a = (const or_keyed *)pa, *b = (const or_keyed *)pb;
    if (a->key != b->key) { return a->key < b->key ? -1 : 1; }
    if (a->idx != b->idx) { return a->idx < b->idx ? -1 : 1; }
    return 0;
}

static int cmp_u64(const void *pa, const void *pb)
{
    uint64_t a = *(const uint64_t *)pa, b = *(const uint64_t *)pb;
    return a < b ? -1 : (a > b ? 1 : 0);
}

/* 64-bit sort key of item `idx` in domain `tag`: first two words of a
 * Philox block under a key derived from the seed. */
static uint64_t perm_key(uint64_t seed, uint64_t idx, uint32_t tag)
{
    uint32_t ctr[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), tag, 0};
    uint32_t key[2] = {(uint32_t)seed ^ 0xA5A5A5A5u, (uint32_t)(seed >> 32) ^ 0x3C3C3C3Cu};
    uint32_t out[4];
    or_philox4x32(ctr, key, out);
    return ((uint64_t)out[0] << 32) | out[1];
}

int64_t or_rmat_finish(int scale, int64_t num_edges, uint64_t seed,
                       int64_t *src, int64_t *dst)
{
    const int64_t n = (int64_t)1 << scale;
    /* flip (edge_list_utils.h:14-24), sort (:27-37), dedup (:40-56) on the
     * packed key src<<32 | dst */
    uint64_t *packed = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(num_edges + 1));
    if (!packed) { return -1; }
    for (int64_t i = 0; i < num_edges; ++i) {
        uint64_t s = (uint64_t)src[i], t = (uint64_t)dst[i];
        if (s > t) { uint64_t x = s; s = t; t = x; }
        packed[i] = (s << 32) | t;
    }
    qsort(packed, (size_t)num_edges, sizeof(uint64_t), cmp_u64);
    int64_t m = 0;
    for (int64_t i = 0; i < num_edges; ++i) {
        if (m == 0 || packed[i] != packed[m - 1]) { packed[m++] = packed[i]; }
    }
    /* relabel (edge_list_utils.h:59-77): the vertex with the k-th smallest
     * key becomes vertex k */
    or_keyed *vk = (or_keyed *)malloc(sizeof(or_keyed) * (size_t)n);
    int64_t *new_id = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    or_keyed *ek = (or_keyed *)malloc(sizeof(or_keyed) * (size_t)(m + 1));
    if (!vk || !new_id || !ek) { free(packed); free(vk); free(new_id); free(ek); return -1; }
    for (int64_t v = 0; v < n; ++v) { vk[v].key = perm_key(seed, (uint64_t)v, 0x52454C42u); vk[v].idx = (uint64_t)v; }
    qsort(vk, (size_t)n, sizeof(or_keyed), cmp_keyed);
    for (int64_t k = 0; k < n; ++k) { new_id[vk[k].idx] = k; }
    /* shuffle (rmat_dataset_dump.cc:57): order edges by a keyed permutation */
    for (int64_t e = 0; e < m; ++e) { ek[e].key = perm_key(seed, (uint64_t)e, 0x53485546u); ek[e].idx = (uint64_t)e; }
    qsort(ek, (size_t)m, sizeof(or_keyed), cmp_keyed);
    for (int64_t k = 0; k < m; ++k) {
        uint64_t p = packed[ek[k].idx];
        src[k] = new_id[p >> 32];
        dst[k] = new_id[p & 0xFFFFFFFFu];
    }
    free(packed);
    free(vk);
    free(new_id);
    free(ek);
    return m;
}

/* The project's grid generator: edge e (horizontal edges row by row, then
 * vertical) survives when the top 53 bits of its Philox key, as a fraction
 * of 2^53, are >= delete_frac.  Returns the number of edges written. */
int64_t or_grid_edges(int64_t rows, int64_t cols, double delete_frac, uint64_t seed,
                      int64_t *src, int64_t *dst)
{
    const int64_t horiz = rows * (cols - 1);
    const int64_t total = horiz + (rows - 1) * cols;
    int64_t m = 0;
    for (int64_t e = 0; e < total; ++e) {
        uint64_t k = perm_key(seed, (uint64_t)e, 0x47524944u);
        double u = (double)(k >> 11) * (1.0 / 9007199254740992.0);
        if (u < delete_frac) { continue; }
        int64_t a, b;
        if (e < horiz) {
            a = (e / (cols - 1)) * cols + e % (cols - 1);
            b = a + 1;
        } else {
            int64_t f = e - horiz;
            a = (f / cols) * cols + f % cols;
            b = a + cols;
        }
        src[m] = a;
        dst[m] = b;
        ++m;
    }
    return m;
}
