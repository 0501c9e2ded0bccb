/* Oracle: plain-C restatement of the reference RelaxMap hot path.
 * TEST INFRASTRUCTURE ONLY (see rmx_oracle.h). Never linked by the product.
 * Citations are file:line in the reference project (uwescience/RelaxMap). */
#include "rmx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ALPHA 0.15              /* Module.h:114 */
#define BETA (1.0 - 0.15)       /* Module.h:116 */

static inline double plogp(double x) { return x > 0.0 ? x * log(x) : 0.0; } /* Module.h:23-25 */

/* ---------------------------------------------------------------- MT19937 */
/* MT19937 (Matsumoto & Nishimura) as bundled with the reference. Seeding from
 * one word is the original 1998 scheme (MersenneTwister.h:172-183): each state
 * word takes the high 16 bits of the seed and of seed*69069, and the seed
 * advances through the linear congruence s -> 69069*s + 1 twice per word. */
void rmxo_mt_seed(rmxo_mt *r, uint32_t seed) {
    for (int i = 0; i < 624; i++) {
        uint32_t hi = seed & 0xffff0000U;
        seed *= 69069U;
        r->state[i] = hi | ((seed & 0xffff0000U) >> 16);
        seed += 1U;
        seed = seed * 69069U + 1U;
    }
    r->left = 0;
    r->next = 624;
}

static void mt_refill(rmxo_mt *r) {
    uint32_t *s = r->state;
    for (int i = 0; i < 624; i++) {
        uint32_t y = (s[i] & 0x80000000U) | (s[(i + 1) % 624] & 0x7fffffffU);
        uint32_t v = s[(i + 397) % 624] ^ (y >> 1);
        if (s[(i + 1) % 624] & 1U) v ^= 0x9908b0dfU;
        s[i] = v;
    }
    r->left = 624;
    r->next = 0;
}

uint32_t rmxo_mt_rand(rmxo_mt *r) {
    if (r->left == 0) mt_refill(r);
    r->left--;
    uint32_t y = r->state[r->next++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680U;
    y ^= (y << 15) & 0xefc60000U;
    return y ^ (y >> 18);
}

/* Uniform integer in [0,n] by masking to the bits n uses and rejecting
 * (MersenneTwister.h:156-169). */
uint32_t rmxo_mt_randint(rmxo_mt *r, uint32_t n) {
    uint32_t used = n;
    used |= used >> 1;
    used |= used >> 2;
    used |= used >> 4;
    used |= used >> 8;
    used |= used >> 16;
    uint32_t i;
    do i = rmxo_mt_rand(r) & used;
    while (i > n);
    return i;
}

/* --------------------------------------------------------------- initiate */
/* calculateSteadyState, Module.cpp:340-469, one thread: teleport part first,
 * then push along out-links into a zeroed scratch, one add per node, then
 * normalise and take the L1 change; stop at 200 iterations or when the change
 * is <= 1e-15 after at least 50 (Module.cpp:460). */
static int steady_state(int N, const int64_t *off, const int32_t *dst, const double *wn, const double *tw,
                        const uint8_t *dangling, double *size) {
    double *prev = (double *)malloc(sizeof(double) * (size_t)N);
    double *added = (double *)malloc(sizeof(double) * (size_t)N);
    for (int i = 0; i < N; i++) prev[i] = 1.0 / N;
    int iter = 0;
    double diff;
    do {
        double dang = 0.0;
        for (int i = 0; i < N; i++)
            if (dangling[i]) dang += prev[i];
        for (int i = 0; i < N; i++) size[i] = (ALPHA + BETA * dang) * tw[i];
        for (int i = 0; i < N; i++) added[i] = 0.0;
        for (int i = 0; i < N; i++)
            for (int64_t j = off[i]; j < off[i + 1]; j++) added[dst[j]] += BETA * wn[j] * prev[i];
        for (int i = 0; i < N; i++) size[i] += added[i];
        double sum = 0.0;
        for (int i = 0; i < N; i++) sum += size[i];
        diff = 0.0;
        for (int i = 0; i < N; i++) {
            size[i] = size[i] / sum;
            diff += fabs(size[i] - prev[i]);
            prev[i] = size[i];
        }
        iter++;
    } while (iter < 200 && (diff > 1.0e-15 || iter < 50));
    free(prev);
    free(added);
    return iter;
}

int rmxo_initiate(int N, const int64_t *off, const int32_t *dst, const double *w, const double *tw, double *p,
                  double *f, double *dsize, double *exitpr, uint8_t *dangling, double *L0, double *all_log_all) {
    /* Module.cpp:228-247: dangling flags; out-weights divided by their row sum */
    for (int i = 0; i < N; i++) {
        dangling[i] = off[i + 1] == off[i];
        double s = 0.0;
        for (int64_t j = off[i]; j < off[i + 1]; j++) s += w[j];
        for (int64_t j = off[i]; j < off[i + 1]; j++) f[j] = w[j] / s;
    }
    int iters = steady_state(N, off, dst, f, tw, dangling, p);
    /* Module.cpp:275-286: edge flow = p_a * normalised weight; dangling size */
    for (int i = 0; i < N; i++) {
        for (int64_t j = off[i]; j < off[i + 1]; j++) f[j] = p[i] * f[j];
        dsize[i] = dangling[i] ? p[i] : 0.0;
    }
    double all = 0.0; /* Module.cpp:295-305 */
    for (int i = 0; i < N; i++) all += plogp(p[i]);
    *all_log_all = all;
    /* singleton modules, Module.cpp:67-99 (exit) and calibrate :474-501 */
    double sel = 0.0, ssl = 0.0, sexit = 0.0;
    for (int i = 0; i < N; i++) {
        double sumf = 0.0;
        for (int64_t j = off[i]; j < off[i + 1]; j++) sumf += f[j];
        double ex = dangling[i] ? (1.0 - tw[i]) * p[i] : ALPHA * (1.0 - tw[i]) * p[i] + BETA * sumf;
        exitpr[i] = ex;
        sel += plogp(ex);
        ssl += plogp(ex + p[i]);
        sexit += ex;
    }
    *L0 = plogp(sexit) - 2.0 * sel + ssl - all;
    return iters;
}

/* ------------------------------------------------------------ code length */
double rmxo_codelength(int N, const int64_t *off, const int32_t *dst, const double *f, const double *p,
                       const double *tw, const double *dsize, const int32_t *part, double all_log_all,
                       double *sum_exit) {
    double *P = calloc((size_t)N, sizeof(double)), *TW = calloc((size_t)N, sizeof(double));
    double *D = calloc((size_t)N, sizeof(double)), *OUT = calloc((size_t)N, sizeof(double));
    int *cnt = calloc((size_t)N, sizeof(int));
    for (int i = 0; i < N; i++) {
        int m = part[i];
        P[m] += p[i];
        TW[m] += tw[i];
        D[m] += dsize[i];
        cnt[m]++;
    }
    /* Module.cpp:2981-2989: members in node order, their out-links leaving m */
    for (int i = 0; i < N; i++)
        for (int64_t j = off[i]; j < off[i + 1]; j++)
            if (part[dst[j]] != part[i]) OUT[part[i]] += f[j];
    double se = 0.0, sel = 0.0, ssl = 0.0;
    for (int m = 0; m < N; m++) {
        if (cnt[m] == 0) continue;
        double ex = ALPHA * (1.0 - TW[m]) * P[m]; /* Module.cpp:2978, 2991 */
        ex += BETA * (OUT[m] + (1.0 - TW[m]) * D[m]);
        se += ex;
        sel += plogp(ex);
        ssl += plogp(ex + P[m]);
    }
    free(P); free(TW); free(D); free(OUT); free(cnt);
    if (sum_exit) *sum_exit = se;
    return plogp(se) - 2.0 * sel + ssl - all_log_all; /* Module.cpp:2999 */
}

/* -------------------------------------------------------------- coarsening */
int rmxo_convert(int N, const int64_t *off, const int32_t *dst, const double *f, const int32_t *part,
                 int32_t *sn_of_mod, int64_t *sn_out_off, int32_t *sn_out_dst, double *sn_out_f,
                 int64_t *sn_in_off, int32_t *sn_in_src, double *sn_in_f, int64_t *n_links) {
    int *cnt = calloc((size_t)N, sizeof(int));
    for (int i = 0; i < N; i++) cnt[part[i]]++;
    int nsn = 0; /* Module.cpp:3015-3022 */
    for (int m = 0; m < N; m++) sn_of_mod[m] = cnt[m] > 0 ? nsn++ : -1;
    /* members per super-node in node order (updateMembersInModule :2900-2901) */
    int64_t *moff = calloc((size_t)nsn + 1, sizeof(int64_t));
    int32_t *mem = malloc(sizeof(int32_t) * (size_t)N);
    for (int i = 0; i < N; i++) moff[sn_of_mod[part[i]] + 1]++;
    for (int s = 0; s < nsn; s++) moff[s + 1] += moff[s];
    int64_t *fill = malloc(sizeof(int64_t) * (size_t)(nsn + 1));
    memcpy(fill, moff, sizeof(int64_t) * (size_t)(nsn + 1));
    for (int i = 0; i < N; i++) mem[fill[sn_of_mod[part[i]]]++] = i;
    /* per super-node: std::map<int,double> keyed by destination SN, first
     * insert then += in member/link order (Module.cpp:3046-3066) */
    double *acc = malloc(sizeof(double) * (size_t)nsn);
    char *seen = calloc((size_t)nsn, 1);
    int32_t *touched = malloc(sizeof(int32_t) * (size_t)nsn);
    int64_t k = 0;
    sn_out_off[0] = 0;
    for (int s = 0; s < nsn; s++) {
        int nt = 0;
        for (int64_t a = moff[s]; a < moff[s + 1]; a++) {
            int u = mem[a];
            for (int64_t j = off[u]; j < off[u + 1]; j++) {
                int t = sn_of_mod[part[dst[j]]];
                if (t == s) continue;
                if (!seen[t]) {
                    seen[t] = 1;
                    acc[t] = f[j];
                    touched[nt++] = t;
                } else {
                    acc[t] += f[j];
                }
            }
        }
        /* map iteration order: ascending destination */
        for (int a = 1; a < nt; a++) {
            int v = touched[a], b = a - 1;
            while (b >= 0 && touched[b] > v) { touched[b + 1] = touched[b]; b--; }
            touched[b + 1] = v;
        }
        for (int a = 0; a < nt; a++) {
            sn_out_dst[k] = touched[a];
            sn_out_f[k] = acc[touched[a]];
            seen[touched[a]] = 0;
            k++;
        }
        sn_out_off[s + 1] = k;
    }
    *n_links = k;
    /* in-links appended in ascending source order (Module.cpp:3071-3075) */
    for (int s = 0; s <= nsn; s++) sn_in_off[s] = 0;
    for (int64_t e = 0; e < k; e++) sn_in_off[sn_out_dst[e] + 1]++;
    for (int s = 0; s < nsn; s++) sn_in_off[s + 1] += sn_in_off[s];
    memcpy(fill, sn_in_off, sizeof(int64_t) * (size_t)(nsn + 1));
    for (int s = 0; s < nsn; s++)
        for (int64_t e = sn_out_off[s]; e < sn_out_off[s + 1]; e++) {
            int64_t q = fill[sn_out_dst[e]]++;
            sn_in_src[q] = s;
            sn_in_f[q] = sn_out_f[e];
        }
    free(cnt); free(moff); free(mem); free(fill); free(acc); free(seen); free(touched);
    return nsn;
}

/* ------------------------------------------------------- move evaluation */
typedef struct {
    int32_t mod;
    double out, in;
} cand_t;

static int cmp_cand(const void *a, const void *b) {
    int32_t x = ((const cand_t *)a)->mod, y = ((const cand_t *)b)->mod;
    return (x > y) - (x < y);
}

/* Aggregate beta * flow to/from each neighbouring module (Module.cpp:1004-1028),
 * per module in link order, out-links first. Returns the number of distinct
 * modules written to c[] (sorted by module id). */
static int aggregate(int u, const int64_t *out_off, const int32_t *out_dst, const double *out_f,
                     const int64_t *in_off, const int32_t *in_src, const double *in_f, const int32_t *mod,
                     cand_t *c) {
    int n = 0;
    for (int64_t j = out_off[u]; j < out_off[u + 1]; j++) c[n++].mod = mod[out_dst[j]];
    for (int64_t j = in_off[u]; j < in_off[u + 1]; j++) c[n++].mod = mod[in_src[j]];
    qsort(c, (size_t)n, sizeof(cand_t), cmp_cand);
    int m = 0;
    for (int a = 0; a < n; a++)
        if (m == 0 || c[m - 1].mod != c[a].mod) { c[m].mod = c[a].mod; c[m].out = 0.0; c[m].in = 0.0; m++; }
    for (int64_t j = out_off[u]; j < out_off[u + 1]; j++) {
        cand_t key = {mod[out_dst[j]], 0, 0};
        cand_t *h = bsearch(&key, c, (size_t)m, sizeof(cand_t), cmp_cand);
        h->out += BETA * out_f[j];
    }
    for (int64_t j = in_off[u]; j < in_off[u + 1]; j++) {
        cand_t key = {mod[in_src[j]], 0, 0};
        cand_t *h = bsearch(&key, c, (size_t)m, sizeof(cand_t), cmp_cand);
        h->in += BETA * in_f[j];
    }
    return m;
}

/* The map-equation change of moving a unit from module 1 to module 2 given the
 * post-move exits (Module.cpp:1106-1115). */
static inline double delta_L(double sum_exit, double new_sum_exit, double ex1, double P1, double ex2, double P2,
                             double nex1, double nP1, double nex2, double nP2) {
    double d_all = plogp(new_sum_exit) - plogp(sum_exit);
    double d_exit = plogp(nex1) + plogp(nex2) - plogp(ex1) - plogp(ex2);
    double d_stay = plogp(nex1 + nP1) + plogp(nex2 + nP2) - plogp(ex1 + P1) - plogp(ex2 + P2);
    return d_all - 2.0 * d_exit + d_stay;
}

void rmxo_evaluate(int nunits, const int64_t *out_off, const int32_t *out_dst, const double *out_f,
                   const int64_t *in_off, const int32_t *in_src, const double *in_f, const double *p,
                   const double *tw, const double *dsize, const double *exitpr, const int32_t *mod,
                   const double *mexit, const double *mP, const double *mTW, const double *mD, double sum_exit,
                   const uint8_t *allow_new, int32_t *best_mod, double *best_delta) {
    int64_t maxdeg = 0;
    for (int u = 0; u < nunits; u++) {
        int64_t d = out_off[u + 1] - out_off[u] + in_off[u + 1] - in_off[u];
        if (d > maxdeg) maxdeg = d;
    }
    cand_t *c = malloc(sizeof(cand_t) * (size_t)(maxdeg + 1));
    for (int u = 0; u < nunits; u++) {
        int nc = aggregate(u, out_off, out_dst, out_f, in_off, in_src, in_f, mod, c);
        int A = mod[u];
        double pu = p[u], tu = tw[u], du = dsize[u], eu = exitpr[u];
        double eA = mexit[A], PA = mP[A], DA = mD[A], TWA = mTW[A];
        /* teleportation / dangling terms, Module.cpp:1047-1061 */
        double outA = (ALPHA * pu + BETA * du) * (TWA - tu);
        double inA = (ALPHA * (PA - pu) + BETA * (DA - du)) * tu;
        for (int a = 0; a < nc; a++) {
            int m = c[a].mod;
            if (m == A) {
                outA = c[a].out + outA;
                inA = c[a].in + inA;
            } else {
                c[a].out += (ALPHA * pu + BETA * du) * mTW[m];
                c[a].in += (ALPHA * mP[m] + BETA * mD[m]) * tu;
            }
        }
        double nexA = eA - eu + outA + inA; /* Module.cpp:1084 */
        double best = 0.0;
        int bm = -1;
        for (int a = 0; a < nc; a++) { /* Module.cpp:1088-1123 */
            int m = c[a].mod;
            if (m == A) continue;
            double em = mexit[m], Pm = mP[m];
            double nexm = em + eu - c[a].out - c[a].in;
            double nse = sum_exit + nexA + nexm - eA - em;
            double d = delta_L(sum_exit, nse, eA, PA, em, Pm, nexA, PA - pu, nexm, Pm + pu);
            if (d < best) { best = d; bm = m; }
        }
        if (allow_new && allow_new[u]) { /* empty module: exit 0, flow 0, teleport terms 0 */
            double nexm = eu;
            double nse = sum_exit + nexA + nexm - eA;
            double d = delta_L(sum_exit, nse, eA, PA, 0.0, 0.0, nexA, PA - pu, nexm, pu);
            if (d < best) { best = d; bm = -2; }
        }
        best_mod[u] = bm;
        best_delta[u] = best;
    }
    free(c);
}

/* --------------------------------------------------- sequential node sweeps */
typedef struct {
    double exit, P, TW, D;
    int members;      /* NumMembers(): live count */
    int listed;       /* members.size(): count at the last updateMembersInModule */
} omod_t;

double rmxo_node_sweeps(int N, const int64_t *off, const int32_t *dst, const double *f, const int64_t *in_off,
                        const int32_t *in_src, const double *in_f, const double *p, const double *tw,
                        const double *dsize, const double *exitpr, const uint8_t *dangling, double L0,
                        uint32_t seed, int prior, double vthresh, double threshold, int max_iter, int32_t *part,
                        int *n_sweeps) {
    rmxo_mt rng;
    rmxo_mt_seed(&rng, seed);
    double vT = -vthresh; /* OmpRelaxmap.cpp:66 */
    omod_t *M = malloc(sizeof(omod_t) * (size_t)N);
    int32_t *empty = malloc(sizeof(int32_t) * (size_t)N);
    int nempty = 0, nmod = N;
    double sum_exit = 0.0, L = L0;
    for (int i = 0; i < N; i++) { /* singletons from initiate, Module.cpp:312-326 */
        part[i] = i;
        M[i].exit = exitpr[i];
        M[i].P = p[i];
        M[i].TW = tw[i];
        M[i].D = dangling[i] ? p[i] : 0.0;
        M[i].members = 1;
        M[i].listed = 1;
        sum_exit += exitpr[i];
    }
    int64_t maxdeg = 0;
    for (int u = 0; u < N; u++) {
        int64_t d = off[u + 1] - off[u] + in_off[u + 1] - in_off[u];
        if (d > maxdeg) maxdeg = d;
    }
    cand_t *c = malloc(sizeof(cand_t) * (size_t)(maxdeg + 2));
    int32_t *order = malloc(sizeof(int32_t) * (size_t)N);
    int32_t *active = malloc(sizeof(int32_t) * (size_t)N);
    uint8_t *isact = calloc((size_t)N, 1);
    int nact = N;
    for (int i = 0; i < N; i++) active[i] = i; /* OmpRelaxmap.cpp:283-288 */
    int iter = 0, stop = 0;
    while (!stop && iter < max_iter) {
        double oldL = L;
        int n = prior ? nact : N;
        for (int i = 0; i < n; i++) order[i] = prior ? active[i] : i;
        for (int i = 0; i < n; i++) { /* Module.cpp:518-525 / :736-743 */
            int t = (int)rmxo_mt_randint(&rng, (uint32_t)(n - 1));
            int tmp = order[i]; order[i] = order[t]; order[t] = tmp;
        }
        for (int i = 0; i < n; i++) {
            int u = order[i];
            int A = part[u];
            int nc = aggregate(u, off, dst, f, in_off, in_src, in_f, part, c);
            double pu = p[u], tu = tw[u], du = dsize[u], eu = exitpr[u];
            double eA = M[A].exit, PA = M[A].P, DA = M[A].D, TWA = M[A].TW;
            double outA = (ALPHA * pu + BETA * du) * (TWA - tu);
            double inA = (ALPHA * (PA - pu) + BETA * (DA - du)) * tu;
            for (int a = 0; a < nc; a++) {
                int m = c[a].mod;
                if (m == A) { outA = c[a].out + outA; inA = c[a].in + inA; }
                else {
                    c[a].out += (ALPHA * pu + BETA * du) * M[m].TW;
                    c[a].in += (ALPHA * M[m].P + BETA * M[m].D) * tu;
                }
            }
            /* empty-module option keyed by the real index emptyModules.back(),
             * gated by the stale member list (Module.cpp:606-611) */
            if (M[A].listed > 1 && nempty > 0) {
                cand_t e = {empty[nempty - 1], 0.0, 0.0};
                int pos = nc;
                while (pos > 0 && c[pos - 1].mod > e.mod) { c[pos] = c[pos - 1]; pos--; }
                c[pos] = e;
                nc++;
            }
            double nexA = eA - eu + outA + inA;
            double best = 0.0, bP1 = 0, bP2 = 0, bE1 = 0, bE2 = 0, bSE = 0;
            int bm = -1;
            for (int a = 0; a < nc; a++) {
                int m = c[a].mod;
                if (m == A) continue;
                double em = M[m].exit, Pm = M[m].P;
                double nexm = em + eu - c[a].out - c[a].in;
                double nse = sum_exit + nexA + nexm - eA - em;
                double d = delta_L(sum_exit, nse, eA, PA, em, Pm, nexA, PA - pu, nexm, Pm + pu);
                if (d < best) { best = d; bm = m; bP1 = PA - pu; bP2 = Pm + pu; bE1 = nexA; bE2 = nexm; bSE = nse; }
            }
            if (best < (prior ? vT : 0.0)) { /* commit, Module.cpp:667-707 / :886-933 */
                int B = bm;
                if (M[B].members == 0) { nempty--; nmod++; }
                part[u] = B;
                M[B].members++;
                M[B].exit = bE2;
                M[B].P = bP2;
                M[B].TW += tu;
                if (dangling[u]) { M[B].D += pu; M[A].D -= pu; }
                M[A].members--;
                M[A].exit = bE1;
                M[A].P = bP1;
                M[A].TW -= tu;
                if (M[A].members == 0) { empty[nempty++] = A; nmod--; }
                sum_exit = bSE;
                L += best;
                if (prior) {
                    for (int64_t j = off[u]; j < off[u + 1]; j++) isact[dst[j]] = 1;
                    for (int64_t j = in_off[u]; j < in_off[u + 1]; j++) isact[in_src[j]] = 1;
                }
            }
        }
        if (prior) { /* Module.cpp:937-943 */
            nact = 0;
            for (int i = 0; i < N; i++)
                if (isact[i]) { active[nact++] = i; isact[i] = 0; }
        }
        iter++;
        if (oldL - L >= 0 && (oldL - L) / log(2.0) < threshold) stop = 1; /* OmpRelaxmap.cpp:328 */
    }
    (void)nmod;
    *n_sweeps = iter;
    free(M); free(empty); free(c); free(order); free(active); free(isact);
    return L;
}
