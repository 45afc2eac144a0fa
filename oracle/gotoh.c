/*
 * oracle/gotoh.c -- CPU restatement of SWhybrid's Smith-Waterman scoring path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/, the smoke
 * entry point and the benchmark's cpu_baseline leg may load it.  The product
 * path (swhybrid_b200/csrc) never calls it.
 *
 * What is restated, with the reference lines it follows (paths inside the
 * SWhybrid project):
 *
 *   cell recurrence      src/AVXKernel.cpp:196-218 (ONE_CELL_UPDATE):
 *                          H = Hdiag + P; H = max(H, F); H = max(H, E);
 *                          S = max(S, H); F -= R; E -= R; N = H; H -= Q;
 *                          E = max(H, E); F = max(H, F)
 *                        with the biased saturating zero of the int8 lanes
 *                        (AVXKernel.cpp:234, 0x80 == score 0), i.e. every
 *                        H/E/F value is floored at 0.  Q = gapOpen+gapExtend
 *                        (Param.h:112, "gapOE"), R = gapExtend.
 *   orientation          query rows x DB columns; E is carried along a query
 *                        row across DB columns (savedE, AVXKernel.cpp:232),
 *                        F down a DB column across query rows (vF[i]).
 *   int8 first pass      score = (u8)S ^ 0x80, scores >= SCORE_LIMIT_7 are
 *                        flagged (AVXKernel.cpp:475-485); SCORE_LIMIT_7 =
 *                        128 - max(matrix) (Worker.cpp:62-70).
 *   int16 recalc         avxCompute16 with the gap costs fixed at 12/2
 *                        (AVXKernel.cpp:914-915), bias 0x8000, saturating at
 *                        65535 (AVXKernel.cpp:977).
 *   query padding        to a multiple of 8 with code 23 (DataPool.cpp:17,
 *                        330-337); code 23 scores 0 (Param.h:8-51 row/col 23).
 *
 * Parity is pinned: tests/golden holds score vectors produced by the
 * reference's own avxCompute/avxCompute16 (compiled from the reference
 * sources by oracle/Makefile into oracle/_ref), and this restatement is
 * checked against them.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* Scalar Gotoh local alignment score, int64, textbook recurrence in the
 * reference's cell order (AVXKernel.cpp:196-218).  mat is 32x32 row-major,
 * indexed mat[query_code * 32 + db_code]. */
int64_t oracle_gotoh(const uint8_t *q, int64_t qlen, const uint8_t *d,
                     int64_t dlen, const int32_t *mat, int32_t gap_oe,
                     int32_t gap_e)
{
    if (qlen <= 0 || dlen <= 0)
        return 0;
    /* H and E of the previous DB column, one entry per query row. */
    int64_t *hcol = (int64_t *)calloc((size_t)qlen, sizeof(int64_t));
    int64_t *ecol = (int64_t *)calloc((size_t)qlen, sizeof(int64_t));
    int64_t best = 0;
    for (int64_t j = 0; j < dlen; ++j) {
        const int dc = d[j] & 31;
        int64_t diag = 0;   /* H(i-1, j-1); row -1 is 0 */
        int64_t f = 0;      /* F entering row 0 of this column */
        for (int64_t i = 0; i < qlen; ++i) {
            int64_t h = diag + mat[(q[i] & 31) * 32 + dc];
            if (h < 0) h = 0;
            int64_t e = ecol[i];
            if (h < f) h = f;
            if (h < e) h = e;
            if (best < h) best = h;
            diag = hcol[i];
            hcol[i] = h;
            int64_t hq = h - gap_oe;
            f -= gap_e; e -= gap_e;
            if (f < 0) f = 0;
            if (e < 0) e = 0;
            if (f < hq) f = hq;
            if (e < hq) e = hq;
            ecol[i] = e;
        }
    }
    free(hcol);
    free(ecol);
    return best;
}

/* Score the reference reports for one DB record after its int8 pass and,
 * when flagged, the RecalcWorker int16 pass (RecalcWorker.cpp:99-268).
 * The int16 pass always uses gap costs 12/2 (AVXKernel.cpp:914-915). */
int64_t oracle_reference_score(const uint8_t *q, int64_t qlen,
                               const uint8_t *d, int64_t dlen,
                               const int32_t *mat, int32_t gap_oe,
                               int32_t gap_e)
{
    int32_t hi = 0;
    for (int k = 0; k < 1024; ++k)
        if (mat[k] > hi) hi = mat[k];
    const int64_t limit7 = 128 - hi;
    int64_t s = oracle_gotoh(q, qlen, d, dlen, mat, gap_oe, gap_e);
    if (s < limit7)
        return s;
    s = oracle_gotoh(q, qlen, d, dlen, mat, 12, 2);
    return s > 65535 ? 65535 : s;
}

/* Score every record of a DB given as a flat residue array plus n+1 offsets.
 * mode 0: exact Gotoh (int64 clipped to int32 range);
 * mode 1: the reference's reported score (int8 pass + int16 recalc). */
void oracle_search(const uint8_t *q, int64_t qlen, const uint8_t *res,
                   const uint64_t *off, int64_t n, const int32_t *mat,
                   int32_t gap_oe, int32_t gap_e, int32_t mode,
                   int32_t threads, int32_t *scores)
{
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
    for (int64_t k = 0; k < n; ++k) {
        const uint8_t *d = res + off[k];
        int64_t dl = (int64_t)(off[k + 1] - off[k]);
        int64_t s = mode ? oracle_reference_score(q, qlen, d, dl, mat, gap_oe, gap_e)
                         : oracle_gotoh(q, qlen, d, dl, mat, gap_oe, gap_e);
        if (s > 2147483647) s = 2147483647;
        scores[k] = (int32_t)s;
    }
}

/* Top-k under the stated tie order: score descending, then record index
 * ascending; records scoring 0 are never reported (ResultList.h:55-79 rejects
 * score <= bottom, and bottom starts at 0).  Returns the number of hits. */
int32_t oracle_topk(const int32_t *scores, int64_t n, int32_t k,
                    int32_t *out_scores, int64_t *out_idx)
{
    int32_t m = 0;
    for (int64_t i = 0; i < n; ++i) {
        int32_t s = scores[i];
        if (s <= 0) continue;
        if (m == k && s <= out_scores[m - 1]) continue;
        int32_t pos = (m < k) ? m : k - 1;
        /* shift down everything strictly smaller (equal scores keep the
         * earlier, i.e. smaller, index first) */
        while (pos > 0 && out_scores[pos - 1] < s) {
            if (pos < k) {
                out_scores[pos] = out_scores[pos - 1];
                out_idx[pos] = out_idx[pos - 1];
            }
            --pos;
        }
        out_scores[pos] = s;
        out_idx[pos] = i;
        if (m < k) ++m;
    }
    return m;
}

/* Traceback of the best local alignment (the reference reports scores only,
 * so this restates the semantics the library's sw_traceback defines; the
 * score it reaches is the Gotoh score above):
 *   H(i,j) = max(0, H(i-1,j-1) + s(q_i, d_j), E(i,j), F(i,j))
 *   E(i,j) = max(E(i,j-1) - e, H(i,j-1) - oe)   (d_j against a gap: 'D')
 *   F(i,j) = max(F(i-1,j) - e, H(i-1,j) - oe)   (q_i against a gap: 'I')
 *   H = 0 on row 0 and column 0, E and F below any reachable value there.
 * End cell: the first cell with the maximal H in column-major order (DB
 * position, then query position).  Walk back from it: in H, stop at H = 0,
 * else prefer the diagonal, then E, then F; in E or F prefer "opened here"
 * over "extended" when both give the value.  out = {score, q_begin, q_end,
 * d_begin, d_end} (0-based, end exclusive); ops in alignment order, codes
 * 0 = M (aligned pair), 1 = I (query residue, gap in DB), 2 = D (DB residue,
 * gap in query).  Returns the number of ops, or -1 if ops_cap is too small. */
int64_t oracle_traceback(const uint8_t *q, int64_t qlen, const uint8_t *d,
                         int64_t dlen, const int32_t *mat, int32_t oe, int32_t e,
                         int64_t *out, uint8_t *ops, int64_t ops_cap)
{
    const int64_t W = dlen + 1;
    const int32_t NEG = -(1 << 28);
    int32_t *H = (int32_t *)calloc((size_t)(qlen + 1) * W, sizeof(int32_t));
    int32_t *E = (int32_t *)malloc((size_t)(qlen + 1) * W * sizeof(int32_t));
    int32_t *F = (int32_t *)malloc((size_t)(qlen + 1) * W * sizeof(int32_t));
    for (int64_t k = 0; k < (qlen + 1) * W; ++k) E[k] = F[k] = NEG;
    int32_t best = 0;
    int64_t bi = 0, bj = 0;
    for (int64_t j = 1; j <= dlen; ++j)
        for (int64_t i = 1; i <= qlen; ++i) {
            const int32_t s = mat[(q[i - 1] & 31) * 32 + (d[j - 1] & 31)];
            int32_t ev = E[i * W + j - 1] - e, eo = H[i * W + j - 1] - oe;
            int32_t fv = F[(i - 1) * W + j] - e, fo = H[(i - 1) * W + j] - oe;
            E[i * W + j] = ev > eo ? ev : eo;
            F[i * W + j] = fv > fo ? fv : fo;
            int32_t h = H[(i - 1) * W + j - 1] + s;
            if (h < E[i * W + j]) h = E[i * W + j];
            if (h < F[i * W + j]) h = F[i * W + j];
            if (h < 0) h = 0;
            H[i * W + j] = h;
            if (h > best) {
                best = h;
                bi = i;
                bj = j;
            }
        }
    out[0] = best;
    out[1] = out[2] = bi;
    out[3] = out[4] = bj;
    int64_t n = 0;
    if (best > 0) {
        int64_t i = bi, j = bj, si = bi, sj = bj;
        int state = 0;   /* 0 H, 1 E, 2 F */
        while (1) {
            if (n >= ops_cap) { n = -1; break; }
            if (state == 0) {
                if (i == 0 || j == 0 || H[i * W + j] == 0) break;
                const int32_t s = mat[(q[i - 1] & 31) * 32 + (d[j - 1] & 31)];
                if (H[i * W + j] == H[(i - 1) * W + j - 1] + s) {
                    ops[n++] = 0;
                    si = i;
                    sj = j;
                    --i;
                    --j;
                } else if (H[i * W + j] == E[i * W + j]) {
                    state = 1;
                } else {
                    state = 2;
                }
            } else if (state == 1) {
                ops[n++] = 2;
                const int open = H[i * W + j - 1] - oe >= E[i * W + j - 1] - e;
                --j;
                state = open ? 0 : 1;
            } else {
                ops[n++] = 1;
                const int open = H[(i - 1) * W + j] - oe >= F[(i - 1) * W + j] - e;
                --i;
                state = open ? 0 : 2;
            }
        }
        if (n > 0) {
            for (int64_t a = 0, b = n - 1; a < b; ++a, --b) {
                uint8_t t = ops[a];
                ops[a] = ops[b];
                ops[b] = t;
            }
        }
        out[1] = si - 1;
        out[3] = sj - 1;
    }
    free(H);
    free(E);
    free(F);
    return n;
}
