/*
 * nsx_ref.c -- C/OpenMP restatement of the reference's NuLnz hot path.
 *
 * TEST INFRASTRUCTURE: this is the timed host-core baseline ("reference
 * restatement") and a second CPU checker.  It is never linked into, loaded
 * by or called from the product library.  The reference itself (Fortran 90 +
 * Intel OpenMP, Windows build) cannot be compiled on this machine: no Fortran
 * compiler is installed.
 *
 * It keeps the reference's data precision and operation order:
 *  - vectors, densities, matrices and the table weights in FP32 (rkw = 4,
 *    src/NuCommon/NuCommon.f90:63); dot products accumulated in FP64 and
 *    stored back in FP32 (dot44, src/NuCommon/ICommon.FI:688-700);
 *  - multiplyx (src/NuLnz/NuCoreX.f90:128-226): OpenMP dynamic schedule over
 *    (output block, J_ar) work items; for every proton operator of the pn
 *    table the active proton rows of each input block are gathered
 *    (single_productm, src/NuCommonX/NuCommonX.f90:745-827) and
 *    T += me * C(:,k) axpy loops of length dar run over every density element
 *    |me| >= 1e-7, the neutron-side product being redone for every proton
 *    operator; then single_product1 (NuCommonX.f90:830-919) transposes T,
 *    applies the proton density with axpy loops of length dbl, transposes back
 *    and scatter-adds into a per-thread full-length accumulator; the thread
 *    accumulators are summed at the end (NuCoreX.f90:221-224);
 *  - multiplya / multiplyb (NuCoreX.f90:76-125, mulmtx NuCommonX.f90:1009-1104):
 *    symmetric segment products, same-parity partitions only;
 *  - standard Lanczos (Lnzs::Lnz_OP, NuCoreX.f90:595-751) with full classical
 *    Gram-Schmidt against every stored vector (lnzort, NuCoreX.f90:753-791),
 *    the vectors kept in RAM rather than in direct-access disk records.
 * The bitmask walks of next_ij/crproj/condim are replaced by the equivalent
 * precomputed (left, right) partition lists in the same traversal order.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "nsx.h"

typedef struct { int pl, pr; int64_t voff; } rblk;
typedef struct { int nb; rblk *b; } rkey;
typedef struct {
  int nspart, minJ2, maxJ2, nJ;
  int *njt;          /* [nJ][nspart] */
  int *poff;         /* [nJ][nspart+1] */
  int *par;
  int nkeys;
  uint64_t *keys;
  rkey *kb;
  float *vals;
  /* like-particle segments: per J list */
  int nseg;
  int *sJ, *snp, *snpr;
  int64_t *soff;
  float *svals;
} rspecies;

typedef struct { int bk, hb; float me; } bent;
typedef struct { int ak; int ne; bent *e; } aent;
typedef struct { int na; aent *a; } witem;

typedef struct ref_handle {
  rspecies A, B;
  int J2, nblocks;
  int *bja, *bjb, *bda, *bdb;
  int64_t *boff, no_state;
  int nwork;
  witem *work;       /* [nblocks][nJa] */
  int nthr;
  float *coefX;      /* [nthr][no_state] */
  size_t bufsz;
  float *buf1, *buf2, *buf3, *buf4;  /* per thread */
  unsigned char *lcoef;
} ref_handle;

static int njt(const rspecies *s, int ip, int J2) {
  if (J2 < s->minJ2 || J2 > s->maxJ2) return 0;
  return s->njt[((J2 - s->minJ2) / 2) * s->nspart + ip];
}
static int poff(const rspecies *s, int ip, int J2) { return s->poff[((J2 - s->minJ2) / 2) * (s->nspart + 1) + ip]; }
static int dimJ(const rspecies *s, int J2) {
  if (J2 < s->minJ2 || J2 > s->maxJ2) return 0;
  return poff(s, s->nspart, J2);
}
static uint64_t pk(int a, int b, int c, int d, int e) {
  return (uint64_t)a | ((uint64_t)b << 8) | ((uint64_t)c << 16) | ((uint64_t)d << 24) | ((uint64_t)e << 32);
}
static int find_key(const rspecies *s, uint64_t k) {
  for (int i = 0; i < s->nkeys; ++i)
    if (s->keys[i] == k) return i;
  return -1;
}

static void load_species(rspecies *s, const nsx_species *in) {
  s->nspart = in->nspart; s->minJ2 = in->minJ2; s->maxJ2 = in->maxJ2;
  s->nJ = (in->maxJ2 - in->minJ2) / 2 + 1;
  s->njt = malloc(sizeof(int) * s->nJ * s->nspart);
  memcpy(s->njt, in->njt, sizeof(int) * s->nJ * s->nspart);
  s->par = malloc(sizeof(int) * s->nspart);
  memcpy(s->par, in->parity, sizeof(int) * s->nspart);
  s->poff = calloc((size_t)s->nJ * (s->nspart + 1), sizeof(int));
  for (int j = 0; j < s->nJ; ++j)
    for (int p = 0; p < s->nspart; ++p)
      s->poff[j * (s->nspart + 1) + p + 1] = s->poff[j * (s->nspart + 1) + p] + s->njt[j * s->nspart + p];
  s->nkeys = in->nkeys;
  s->keys = malloc(sizeof(uint64_t) * (s->nkeys + 1));
  s->kb = calloc(s->nkeys + 1, sizeof(rkey));
  int64_t nv = in->nkeys ? in->val_off[in->nkeys] : 0;
  s->vals = malloc(sizeof(float) * (nv + 1));
  for (int64_t i = 0; i < nv; ++i) s->vals[i] = (float)in->vals[i];
  for (int k = 0; k < in->nkeys; ++k) {
    const uint8_t *b = in->keys + 8 * k;
    s->keys[k] = pk(b[0], b[1], b[2], b[3], b[4]);
    int cnt = 0;
    for (int r = 0; r < s->nspart; ++r)
      for (int l = 0; l < s->nspart; ++l)
        if ((in->masks[((size_t)k * s->nspart + r) * in->words + l / 32] >> (l % 32)) & 1u) ++cnt;
    s->kb[k].nb = cnt;
    s->kb[k].b = malloc(sizeof(rblk) * (cnt + 1));
    int64_t v = in->val_off[k];
    cnt = 0;
    for (int r = 0; r < s->nspart; ++r)
      for (int l = 0; l < s->nspart; ++l)
        if ((in->masks[((size_t)k * s->nspart + r) * in->words + l / 32] >> (l % 32)) & 1u) {
          s->kb[k].b[cnt].pl = l; s->kb[k].b[cnt].pr = r; s->kb[k].b[cnt].voff = v;
          v += (int64_t)njt(s, l, b[0]) * njt(s, r, b[1]);
          ++cnt;
        }
  }
  s->nseg = in->nseg;
  s->sJ = malloc(sizeof(int) * (s->nseg + 1)); s->snp = malloc(sizeof(int) * (s->nseg + 1));
  s->snpr = malloc(sizeof(int) * (s->nseg + 1)); s->soff = malloc(sizeof(int64_t) * (s->nseg + 1));
  int64_t ns = in->nseg ? in->seg_off[in->nseg] : 0;
  s->svals = malloc(sizeof(float) * (ns + 1));
  for (int g = 0; g < s->nseg; ++g) {
    s->sJ[g] = in->seg_J2[g]; s->snp[g] = in->seg_np[g] - 1; s->snpr[g] = in->seg_npr[g] - 1; s->soff[g] = in->seg_off[g];
  }
  for (int64_t i = 0; i < ns; ++i) s->svals[i] = (float)in->seg_vals[i];
}

/* Racah weight, as src/NuLnz/NuCoreX.f90:1114-1126 (own 6-j, Racah formula) */
static double fh(int n2) { double f = 1; for (int i = 2; i <= n2 / 2; ++i) f *= i; return f; }
static int tri(int a, int b, int c) { return abs(a - b) <= c && c <= a + b && ((a + b + c) % 2 == 0); }
static double dl(int a, int b, int c) { return fh(a + b - c) * fh(a - b + c) * fh(-a + b + c) / fh(a + b + c + 2); }
static double sixj(int a, int b, int c, int d, int e, int f) {
  if (!tri(a, b, c) || !tri(a, e, f) || !tri(d, b, f) || !tri(d, e, c)) return 0;
  double pre = sqrt(dl(a, b, c) * dl(a, e, f) * dl(d, b, f) * dl(d, e, c));
  int lo = a + b + c, t;
  if (a + e + f > lo) lo = a + e + f; if (d + b + f > lo) lo = d + b + f; if (d + e + c > lo) lo = d + e + c;
  int hi = a + b + d + e; if (b + c + e + f < hi) hi = b + c + e + f; if (a + c + d + f < hi) hi = a + c + d + f;
  double s = 0;
  for (t = lo; t <= hi; t += 2)
    s += ((t / 2) % 2 ? -1.0 : 1.0) * fh(t + 2) /
         (fh(t - a - b - c) * fh(t - a - e - f) * fh(t - d - b - f) * fh(t - d - e - c) * fh(a + b + d + e - t) *
          fh(b + c + e + f - t) * fh(a + c + d + f - t));
  return pre * s;
}
static double racahs(int jal, int jbl, int jar, int jbr, int J, int lam) {
  double w = (((jal + jbl + jar + jbr) / 2) % 2 ? -1.0 : 1.0) * sixj(jal, jbl, J, jbr, jar, lam);
  if (w == 0) return 0;
  return (((jal + jbr - J - lam) / 2) % 2 ? -1.0 : 1.0) * w * sqrt(lam + 1.0);
}

ref_handle *ref_create(const nsx_problem *p) {
  ref_handle *h = calloc(1, sizeof(ref_handle));
  load_species(&h->A, &p->a);
  load_species(&h->B, &p->b);
  h->J2 = p->J2;
  rspecies *A = &h->A, *B = &h->B;
  int J2 = p->J2, nb = 0;
  for (int ja = A->minJ2; ja <= A->maxJ2; ja += 2) {
    int lo = abs(ja - J2) > B->minJ2 ? abs(ja - J2) : B->minJ2, hi = ja + J2 < B->maxJ2 ? ja + J2 : B->maxJ2;
    lo += (lo - B->minJ2) % 2;
    for (int jb = lo; jb <= hi; jb += 2) ++nb;
  }
  h->nblocks = nb;
  h->bja = malloc(sizeof(int) * nb); h->bjb = malloc(sizeof(int) * nb);
  h->bda = malloc(sizeof(int) * nb); h->bdb = malloc(sizeof(int) * nb);
  h->boff = malloc(sizeof(int64_t) * (nb + 1));
  nb = 0;
  int64_t off = 0;
  for (int ja = A->minJ2; ja <= A->maxJ2; ja += 2) {
    int lo = abs(ja - J2) > B->minJ2 ? abs(ja - J2) : B->minJ2, hi = ja + J2 < B->maxJ2 ? ja + J2 : B->maxJ2;
    lo += (lo - B->minJ2) % 2;
    for (int jb = lo; jb <= hi; jb += 2) {
      h->bja[nb] = ja; h->bjb[nb] = jb; h->bda[nb] = dimJ(A, ja); h->bdb[nb] = dimJ(B, jb);
      h->boff[nb] = off; off += (int64_t)h->bda[nb] * h->bdb[nb]; ++nb;
    }
  }
  h->boff[nb] = off;
  h->no_state = off;
  h->lcoef = calloc(off, 1);
  for (int k = 0; k < nb; ++k) {
    int64_t n = h->boff[k];
    for (int q = 0; q < B->nspart; ++q)
      for (int kb = 0; kb < njt(B, q, h->bjb[k]); ++kb)
        for (int pp = 0; pp < A->nspart; ++pp)
          for (int ka = 0; ka < njt(A, pp, h->bja[k]); ++ka, ++n)
            h->lcoef[n] = (p->parity == 0 || A->par[pp] * B->par[q] == p->parity);
  }
  /* drdbh: for each (output block, J_ar): proton operators and their (b, h, me) lists */
  h->nwork = nb * A->nJ;
  h->work = calloc(h->nwork, sizeof(witem));
  for (int bsc = 0; bsc < nb; ++bsc) {
    int jal = h->bja[bsc], jbl = h->bjb[bsc];
    for (int ja = 0; ja < A->nJ; ++ja) {
      int jar = A->minJ2 + 2 * ja;
      witem *w = &h->work[bsc * A->nJ + ja];
      w->a = calloc(A->nkeys + 1, sizeof(aent));
      for (int ak = 0; ak < A->nkeys; ++ak) {
        uint64_t key = A->keys[ak];
        if ((int)(key & 255) != jal || (int)((key >> 8) & 255) != jar) continue;
        int sal = (key >> 16) & 255, sar = (key >> 24) & 255, lam = (key >> 32) & 255;
        aent ae = {ak, 0, malloc(sizeof(bent) * (B->nkeys + 1))};
        for (int hb = 0; hb < nb; ++hb) {
          if (h->bja[hb] != jar) continue;
          int jbr = h->bjb[hb];
          double rc = racahs(jal, jbl, jar, jbr, J2, lam);
          if (rc == 0) continue;
          for (int bk = 0; bk < B->nkeys; ++bk) {
            uint64_t kb = B->keys[bk];
            if ((int)(kb & 255) != jbl || (int)((kb >> 8) & 255) != jbr || (int)((kb >> 32) & 255) != lam) continue;
            int sbl = (kb >> 16) & 255, sbr = (kb >> 24) & 255;
            double v = 0; int found = 0;
            uint64_t ok = pk(sal, sar, sbl, sbr, lam);
            for (int o = 0; o < p->nop; ++o) {
              const uint8_t *q = p->op_keys + 8 * o;
              if (pk(q[0], q[1], q[2], q[3], q[4]) == ok) { v = p->op_vals[o]; found = 1; break; }
            }
            if (!found || fabs(v) < 1e-10) continue;
            float me = (float)(v * p->renorm) * (float)rc;
            if (me == 0.0f) continue;
            ae.e[ae.ne].bk = bk; ae.e[ae.ne].hb = hb; ae.e[ae.ne].me = me; ++ae.ne;
          }
        }
        if (ae.ne) w->a[w->na++] = ae; else free(ae.e);
      }
    }
  }
  h->nthr = omp_get_max_threads();
  int maxda = 0, maxdb = 0;
  for (int j = A->minJ2; j <= A->maxJ2; j += 2) if (dimJ(A, j) > maxda) maxda = dimJ(A, j);
  for (int j = B->minJ2; j <= B->maxJ2; j += 2) if (dimJ(B, j) > maxdb) maxdb = dimJ(B, j);
  h->bufsz = (size_t)maxda * maxdb;
  h->coefX = malloc(sizeof(float) * h->nthr * off);
  h->buf1 = malloc(sizeof(float) * h->nthr * h->bufsz);
  h->buf2 = malloc(sizeof(float) * h->nthr * h->bufsz);
  h->buf3 = malloc(sizeof(float) * h->nthr * h->bufsz);
  h->buf4 = malloc(sizeof(float) * h->nthr * h->bufsz);
  return h;
}

int64_t ref_dim(const ref_handle *h) { return h->no_state; }
int ref_nthreads(const ref_handle *h) { return h->nthr; }

/* multiplyx: pn term, overwrites out */
static void multiplyx(ref_handle *h, const float *in, float *out) {
  rspecies *A = &h->A, *B = &h->B;
  const int64_t N = h->no_state;
#pragma omp parallel
  {
    int t = omp_get_thread_num();
    float *X = h->coefX + (size_t)t * N;
    memset(X, 0, sizeof(float) * N);
    float *T = h->buf3 + (size_t)t * h->bufsz, *G = h->buf1 + (size_t)t * h->bufsz;
    float *T2 = h->buf2 + (size_t)t * h->bufsz, *O = h->buf4 + (size_t)t * h->bufsz;
    int *arow = malloc(sizeof(int) * (A->nspart + 1)), *acol = malloc(sizeof(int) * (A->nspart + 1));
    int *bcol = malloc(sizeof(int) * (B->nspart + 1));
#pragma omp for schedule(dynamic, 1)
    for (int wi = 0; wi < h->nwork; ++wi) {
      witem *w = &h->work[wi];
      int bsc = wi / A->nJ, jar = A->minJ2 + 2 * (wi % A->nJ);
      int jal = h->bja[bsc], jbl = h->bjb[bsc];
      for (int ai = 0; ai < w->na; ++ai) {
        aent *ae = &w->a[ai];
        rkey *ka = &A->kb[ae->ak];
        /* crproj/condim: active right (lvac) and left (lvar) proton partitions; output columns (lvbr) */
        for (int q = 0; q < A->nspart; ++q) { acol[q] = -1; arow[q] = -1; }
        for (int q = 0; q < B->nspart; ++q) bcol[q] = -1;
        for (int i = 0; i < ka->nb; ++i) { acol[ka->b[i].pr] = 0; arow[ka->b[i].pl] = 0; }
        int dar = 0, dal = 0, dbl = 0;
        for (int q = 0; q < A->nspart; ++q) if (acol[q] >= 0) { acol[q] = dar; dar += njt(A, q, jar); }
        for (int q = 0; q < A->nspart; ++q) if (arow[q] >= 0) { arow[q] = dal; dal += njt(A, q, jal); }
        for (int e = 0; e < ae->ne; ++e) {
          rkey *kb = &B->kb[ae->e[e].bk];
          for (int i = 0; i < kb->nb; ++i) bcol[kb->b[i].pl] = 0;
        }
        for (int q = 0; q < B->nspart; ++q) if (bcol[q] >= 0) { bcol[q] = dbl; dbl += njt(B, q, jbl); }
        if (dar == 0 || dbl == 0) continue;
        memset(T, 0, sizeof(float) * (size_t)dar * dbl);
        /* single_productm: per input block, gather active rows, axpy over density elements */
        for (int e = 0; e < ae->ne; ++e) {
          int hb = ae->e[e].hb;
          if (e == 0 || ae->e[e - 1].hb != hb) {
            /* gather BUFFER1: all columns of C_h, active proton rows */
            int dbr = h->bdb[hb], da = h->bda[hb];
            const float *C = in + h->boff[hb];
            for (int c = 0; c < dbr; ++c)
              for (int q = 0; q < A->nspart; ++q)
                if (acol[q] >= 0) {
                  int n = njt(A, q, jar);
                  memcpy(G + (size_t)c * dar + acol[q], C + (size_t)c * da + poff(A, q, jar), sizeof(float) * n);
                }
          }
          rkey *kb = &B->kb[ae->e[e].bk];
          float me0 = ae->e[e].me;
          int jbr = h->bjb[hb];
          for (int i = 0; i < kb->nb; ++i) {
            int ql = kb->b[i].pl, qr = kb->b[i].pr;
            int nl = njt(B, ql, jbl), nr = njt(B, qr, jbr);
            const float *rv = B->vals + kb->b[i].voff;
            for (int k = 0; k < nr; ++k) {
              const float *src = G + (size_t)(poff(B, qr, jbr) + k) * dar;
              for (int l = 0; l < nl; ++l) {
                float me = rv[l + nl * k] * me0;
                if (fabsf(me) < 1e-7f) continue;
                float *dst = T + (size_t)(bcol[ql] + l) * dar;
                for (int r = 0; r < dar; ++r) dst[r] += me * src[r];
              }
            }
          }
        }
        /* single_product1: transpose, proton density, transpose back, scatter-add */
        for (int c = 0; c < dbl; ++c)
          for (int r = 0; r < dar; ++r) T2[(size_t)r * dbl + c] = T[(size_t)c * dar + r];
        memset(O, 0, sizeof(float) * (size_t)dal * dbl);
        for (int i = 0; i < ka->nb; ++i) {
          int pl = ka->b[i].pl, pr = ka->b[i].pr;
          int nl = njt(A, pl, jal), nr = njt(A, pr, jar);
          const float *rv = A->vals + ka->b[i].voff;
          for (int k = 0; k < nr; ++k) {
            const float *src = T2 + (size_t)(acol[pr] + k) * dbl;
            for (int l = 0; l < nl; ++l) {
              float me = rv[l + nl * k];
              if (fabsf(me) < 1e-7f) continue;
              float *dst = O + (size_t)(arow[pl] + l) * dbl;
              for (int c = 0; c < dbl; ++c) dst[c] += me * src[c];
            }
          }
        }
        float *Xo = X + h->boff[bsc];
        int da = h->bda[bsc];
        for (int q = 0; q < B->nspart; ++q) {
          if (bcol[q] < 0) continue;
          for (int kb2 = 0; kb2 < njt(B, q, jbl); ++kb2) {
            int c = bcol[q] + kb2, col = poff(B, q, jbl) + kb2;
            for (int pq = 0; pq < A->nspart; ++pq) {
              if (arow[pq] < 0) continue;
              int n = njt(A, pq, jal);
              float *dst = Xo + (size_t)col * da + poff(A, pq, jal);
              for (int l = 0; l < n; ++l) dst[l] += O[(size_t)(arow[pq] + l) * dbl + c];
            }
          }
        }
      }
    }
    free(arow); free(acol); free(bcol);
  }
  /* coefL = sum over threads (NuCoreX.f90:221-224) */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    float s = 0;
    for (int t = 0; t < h->nthr; ++t) s += h->coefX[(size_t)t * N + i];
    out[i] = s;
  }
}

/* multiplya + multiplyb: out += H_pp C + C H_nn, symmetric segments (mulmtx) */
static void multiplyab(ref_handle *h, const float *in, float *out) {
  rspecies *A = &h->A, *B = &h->B;
#pragma omp parallel for schedule(dynamic, 1)
  for (int bsc = 0; bsc < h->nblocks; ++bsc) {
    int ja = h->bja[bsc], jb = h->bjb[bsc], da = h->bda[bsc], db = h->bdb[bsc];
    if (da == 0 || db == 0) continue;
    const float *C = in + h->boff[bsc];
    float *Y = out + h->boff[bsc];
    for (int g = 0; g < A->nseg; ++g) {
      if (A->sJ[g] != ja) continue;
      int i = A->snp[g], j = A->snpr[g];
      if (A->par[i] != A->par[j]) continue;
      int ni = njt(A, i, ja), nj = njt(A, j, ja);
      const float *M = A->svals + A->soff[g];   /* M[kr + nj*kl] = H[(i,kl),(j,kr)] */
      for (int c = 0; c < db; ++c)
        for (int kl = 0; kl < ni; ++kl)
          for (int kr = 0; kr < nj; ++kr) {
            float me = M[kr + (size_t)nj * kl];
            if (me == 0.0f) continue;
            Y[(size_t)c * da + poff(A, i, ja) + kl] += me * C[(size_t)c * da + poff(A, j, ja) + kr];
            if (i != j) Y[(size_t)c * da + poff(A, j, ja) + kr] += me * C[(size_t)c * da + poff(A, i, ja) + kl];
          }
    }
    for (int g = 0; g < B->nseg; ++g) {
      if (B->sJ[g] != jb) continue;
      int i = B->snp[g], j = B->snpr[g];
      if (B->par[i] != B->par[j]) continue;
      int ni = njt(B, i, jb), nj = njt(B, j, jb);
      const float *M = B->svals + B->soff[g];
      for (int kl = 0; kl < ni; ++kl)
        for (int kr = 0; kr < nj; ++kr) {
          float me = M[kr + (size_t)nj * kl];
          if (me == 0.0f) continue;
          float *yl = Y + (size_t)(poff(B, i, jb) + kl) * da, *yr = Y + (size_t)(poff(B, j, jb) + kr) * da;
          const float *cl = C + (size_t)(poff(B, i, jb) + kl) * da, *cr = C + (size_t)(poff(B, j, jb) + kr) * da;
          for (int r = 0; r < da; ++r) yl[r] += me * cr[r];
          if (i != j)
            for (int r = 0; r < da; ++r) yr[r] += me * cl[r];
        }
    }
  }
}

void ref_matvec(ref_handle *h, const float *in, float *out) {
  multiplyx(h, in, out);
  multiplyab(h, in, out);
}

static double dot44(const float *a, const float *b, int64_t n) {
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; ++i) s += (double)a[i] * (double)b[i];
  return s;
}

/* Standard Lanczos (NuCoreX.f90:595-707) for nsteps iterations after npre power
 * pre-iterations, vectors in RAM.  Writes alpha/beta (nsteps each) and returns
 * the wall seconds spent in the steps (pre-iterations in pre_seconds; the part of
 * the steps spent in the Gram-Schmidt loop against the stored vectors in
 * cgs_seconds, so that its cost per stored vector is measured, not inferred). */
double ref_lanczos(ref_handle *h, int npre, int nsteps, uint64_t seed, double *alpha, double *beta,
                   double *pre_seconds, double *cgs_seconds) {
  const int64_t N = h->no_state;
  float *V = malloc(sizeof(float) * N * (size_t)(nsteps + 1));
  memset(V, 0, sizeof(float) * N * (size_t)(nsteps + 1));  /* first touch outside the timed steps */
  float *L = malloc(sizeof(float) * N), *R = malloc(sizeof(float) * N), *Tv = malloc(sizeof(float) * N);
  uint64_t z = seed ? seed : 5;
  for (int64_t i = 0; i < N; ++i) {
    z = z * 6364136223846793005ull + 1442695040888963407ull;
    float x = (float)((z >> 11) * (1.0 / 9007199254740992.0));
    L[i] = h->lcoef[i] ? 0.5f - x : 0.0f;
  }
  double t0 = omp_get_wtime();
  float ovl = (float)(1.0 / sqrt(dot44(L, L, N)));
  for (int64_t i = 0; i < N; ++i) R[i] = ovl * L[i];
  for (int it = 0; it < npre; ++it) {
    ref_matvec(h, R, L);
    ovl = (float)(1.0 / sqrt(dot44(L, L, N)));
    for (int64_t i = 0; i < N; ++i) R[i] = ovl * L[i];
  }
  double t1 = omp_get_wtime();
  if (pre_seconds) *pre_seconds = t1 - t0;
  memcpy(V, R, sizeof(float) * N);
  float b = 0;
  double tcgs = 0;
  for (int it = 0; it < nsteps; ++it) {
    ref_matvec(h, R, L);
    if (it) {
#pragma omp parallel for
      for (int64_t i = 0; i < N; ++i) L[i] -= b * Tv[i];
    }
    memcpy(Tv, R, sizeof(float) * N);
    float a = (float)dot44(R, L, N);
#pragma omp parallel for
    for (int64_t i = 0; i < N; ++i) L[i] -= a * R[i];
    /* lnzort: classical Gram-Schmidt against all stored vectors (NuCoreX.f90:766-778) */
    const double tg0 = omp_get_wtime();
    memcpy(R, L, sizeof(float) * N);
    for (int j = 0; j <= it; ++j) {
      const float *vj = V + (size_t)j * N;
      float o = 0;
      double s = 0;
#pragma omp parallel for reduction(+ : s)
      for (int64_t i = 0; i < N; ++i) s += (double)R[i] * vj[i];
      o = (float)s;
#pragma omp parallel for
      for (int64_t i = 0; i < N; ++i) L[i] -= o * vj[i];
    }
    tcgs += omp_get_wtime() - tg0;
    b = (float)sqrt(dot44(L, L, N));
    alpha[it] = a;
    beta[it] = b;
    float inv = b > 0 ? 1.0f / b : 0.0f;
    for (int64_t i = 0; i < N; ++i) R[i] = inv * L[i];
    memcpy(V + (size_t)(it + 1) * N, R, sizeof(float) * N);
  }
  double t2 = omp_get_wtime();
  if (cgs_seconds) *cgs_seconds = tcgs;
  free(V); free(L); free(R); free(Tv);
  return t2 - t1;
}

/* Number of eigenvalues below x of the symmetric tridiagonal matrix (diagonal a[0..n),
 * off-diagonal b[1..n)), by the Sturm sequence of its LDL^T factorisation (Golub & Van Loan,
 * Matrix Computations, section 8.4.1). */
static int sturm_count(const double *a, const double *b, int n, double x) {
  int cnt = 0;
  double q = a[0] - x;
  if (q < 0) ++cnt;
  for (int i = 1; i < n; ++i) {
    if (q == 0.0) q = 1e-300;
    q = a[i] - x - b[i] * b[i] / q;
    if (q < 0) ++cnt;
  }
  return cnt;
}
/* The k lowest eigenvalues of that matrix by bisection (out[0..k) ascending). */
static void tri_lowest(const double *a, const double *b, int n, int k, double *out) {
  double lo = a[0], hi = a[0];
  for (int i = 0; i < n; ++i) {
    double r = (i > 0 ? fabs(b[i]) : 0.0) + (i + 1 < n ? fabs(b[i + 1]) : 0.0);
    if (a[i] - r < lo) lo = a[i] - r;
    if (a[i] + r > hi) hi = a[i] + r;
  }
  const double eps = 1e-13 * (fabs(lo) + fabs(hi) + 1.0);
  for (int j = 0; j < k && j < n; ++j) {
    double l = lo, u = hi;
    while (u - l > eps) {
      double m = 0.5 * (l + u);
      if (sturm_count(a, b, n, m) > j) u = m; else l = m;
    }
    out[j] = 0.5 * (l + u);
  }
}

/* A complete solve by the reference's standard Lanczos (NuLnz Lnz_OP, NuCoreX.f90:595-751):
 * seeded start on the allowed entries, npre power pre-iterations, the three-term recurrence
 * with classical Gram-Schmidt against every stored vector (vectors in RAM), breakdown restart
 * below restart_limit, and its stopping rule: the first test after first_iter steps, then
 * every inc_iter + 1 steps, until the lowest nlev + 1 Ritz values change by less than
 * level_limit between tests, or noiter steps.  Writes the lowest nlev Ritz values and the
 * step count; returns the wall seconds of the whole solve (pre-iterations included). */
double ref_solve(ref_handle *h, int npre, int nlev, int first_iter, int inc_iter, int noiter, double level_limit,
                 uint64_t seed, double *evals, int *iterations) {
  const int64_t N = h->no_state;
  float *V = malloc(sizeof(float) * N * (size_t)(noiter + 1));
  memset(V, 0, sizeof(float) * N * (size_t)(noiter + 1));
  float *L = malloc(sizeof(float) * N), *R = malloc(sizeof(float) * N), *Tv = malloc(sizeof(float) * N);
  double *al = calloc((size_t)noiter + 2, sizeof(double)), *be = calloc((size_t)noiter + 2, sizeof(double));
  double *prev = calloc((size_t)nlev + 2, sizeof(double)), *cur = calloc((size_t)nlev + 2, sizeof(double));
  int64_t nallowed = 0;
  for (int64_t i = 0; i < N; ++i) nallowed += h->lcoef[i] ? 1 : 0;
  uint64_t z = seed ? seed : 5;
  for (int64_t i = 0; i < N; ++i) {
    z = z * 6364136223846793005ull + 1442695040888963407ull;
    float x = (float)((z >> 11) * (1.0 / 9007199254740992.0));
    L[i] = h->lcoef[i] ? 0.5f - x : 0.0f;
  }
  double t0 = omp_get_wtime();
  float ovl = (float)(1.0 / sqrt(dot44(L, L, N)));
  for (int64_t i = 0; i < N; ++i) R[i] = ovl * L[i];
  for (int it = 0; it < npre; ++it) {
    ref_matvec(h, R, L);
    ovl = (float)(1.0 / sqrt(dot44(L, L, N)));
    for (int64_t i = 0; i < N; ++i) R[i] = ovl * L[i];
  }
  memcpy(V, R, sizeof(float) * N);
  float b = 0;
  int it = 0, next_test = first_iter, done = 0;
  const int nk = nlev + 1;
  for (; it < noiter && !done; ++it) {
    ref_matvec(h, R, L);
    if (it) {
#pragma omp parallel for
      for (int64_t i = 0; i < N; ++i) L[i] -= b * Tv[i];
    }
    memcpy(Tv, R, sizeof(float) * N);
    float a = (float)dot44(R, L, N);
    al[it] = a;
    if (it + 1 >= nallowed) { ++it; break; }   /* Krylov space complete */
#pragma omp parallel for
    for (int64_t i = 0; i < N; ++i) L[i] -= a * R[i];
    memcpy(R, L, sizeof(float) * N);
    for (int j = 0; j <= it; ++j) {
      const float *vj = V + (size_t)j * N;
      double s = 0;
#pragma omp parallel for reduction(+ : s)
      for (int64_t i = 0; i < N; ++i) s += (double)R[i] * vj[i];
      const float o = (float)s;
#pragma omp parallel for
      for (int64_t i = 0; i < N; ++i) L[i] -= o * vj[i];
    }
    double nb = sqrt(dot44(L, L, N));
    if (nb > 1e-7) {
      b = (float)nb;
    } else {   /* breakdown: a random direction orthogonal to the stored vectors, zero coupling */
      for (int64_t i = 0; i < N; ++i) {
        z = z * 6364136223846793005ull + 1442695040888963407ull;
        L[i] = h->lcoef[i] ? (float)(1000.0 * ((z >> 11) * (1.0 / 9007199254740992.0))) * L[i] : 0.0f;
      }
      for (int j = 0; j <= it; ++j) {
        const float *vj = V + (size_t)j * N;
        const float o = (float)dot44(L, vj, N);
        for (int64_t i = 0; i < N; ++i) L[i] -= o * vj[i];
      }
      nb = sqrt(dot44(L, L, N));
      if (nb < 1e-7) { ++it; break; }
      b = 0.0f;
    }
    be[it + 1] = b;
    const float inv = (float)(1.0 / nb);
    for (int64_t i = 0; i < N; ++i) R[i] = inv * L[i];
    memcpy(V + (size_t)(it + 1) * N, R, sizeof(float) * N);
    if (it + 1 == next_test) {
      tri_lowest(al, be, it + 1, nk, cur);
      done = 1;
      for (int j = 0; j < nk && j < it + 1; ++j)
        if (fabs(cur[j] - prev[j]) > level_limit) done = 0;
      memcpy(prev, cur, sizeof(double) * (size_t)nk);
      next_test = it + 1 + inc_iter + 1;
    }
  }
  double t1 = omp_get_wtime();
  tri_lowest(al, be, it, nlev, evals);
  *iterations = it;
  free(V); free(L); free(R); free(Tv); free(al); free(be); free(prev); free(cur);
  return t1 - t0;
}

void ref_destroy(ref_handle *h) {
  if (!h) return;
  /* process-lifetime baseline objects: release the large buffers */
  free(h->coefX); free(h->buf1); free(h->buf2); free(h->buf3); free(h->buf4); free(h->lcoef);
  free(h);
}
