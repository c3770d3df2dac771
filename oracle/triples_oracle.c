/*
 * CPU oracle for the CCSD(T) perturbative-triples energy and its adjoint.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * pyscfad_b200/csrc; only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py may load it.  The product never calls it.
 *
 * It restates, in plain FP64 loops (no BLAS), the algorithm of
 *   pyscfad/cc/ccsd_t_slow.py:29-125        (energy formula, a>=b>=c weights)
 *   pyscfadlib/pyscfadlib/vjp/cc/ccsd_t.c:121-152   (get_wv: which t2/ovoo
 *        elements each W and V term reads)
 *   pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:9-329 (adjoint: z_bar, d_bar,
 *        W_bar = e*z*d + r3^T(z_bar), mo_energy_bar, per-permutation
 *        scatter into the ERI / amplitude gradients)
 *
 * Layouts are the reference's canonical ones (C order, FP64):
 *   mo_energy[n], t1[o,v], t2[o,o,v,v], ovoo[o,v,o,o], ovov[o,v,o,v],
 *   ovvv[o,v,v,v] (unpacked), fvo[v,o] = fock[o:,:o].
 * Gradients are returned w.r.t. each array as an independent tensor, with
 * exactly the element attribution of the reference's C VJP:
 *   w^{pqr}_{xyz} = sum_f ovvv[p,x,f,y] t2[r,q,z,f]
 *                 - sum_m ovoo[p,x,m,q] t2[r,m,z,y]
 *   v^{pqr}_{xyz} = ovov[p,x,q,y] t1[r,z] + t2[q,p,y,x] fvo[z,r]
 * (ccsd_t.c:162-175: the ooov GEMM reads t2T[c,b] = t2[k,m,c,b] and the V
 * term reads t2T[b,a] = t2[j,i,b,a]).
 *
 * E(T) = 2 sum_{a>=b>=c} s^-1 sum_{ijk} WW z / D,  z = r3(WW + VV/2),
 * s = 6 if a==c, 2 if a==b or b==c, else 1 (ccsd_t_slow.py:48-58,84-124).
 * Jobs are restricted to a in [a0,a1) so callers can take slices.
 */
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define IDX4(a, b, c, d, n1, n2, n3) ((((size_t)(a) * (n1) + (b)) * (n2) + (c)) * (n3) + (d))

typedef struct {
    int o, v;
    const double *mo_energy, *t1, *t2, *ovoo, *ovov, *ovvv, *fvo;
} Inputs;

typedef struct {
    double *mo_energy_bar, *t1_bar, *t2_bar, *ovoo_bar, *ovov_bar, *ovvv_bar, *fvo_bar;
} Grads;

/* raw w for one virtual ordering (x,y,z): out[p*o*o+q*o+r] */
static void raw_w(const Inputs *in, int x, int y, int z, double *out)
{
    const int o = in->o, v = in->v;
    for (int p = 0; p < o; p++)
    for (int q = 0; q < o; q++)
    for (int r = 0; r < o; r++) {
        double s = 0;
        const double *a = in->ovvv + IDX4(p, x, 0, y, v, v, v);   /* stride v over f */
        const double *b = in->t2 + IDX4(r, q, z, 0, o, v, v);     /* contiguous f */
        for (int f = 0; f < v; f++) s += a[(size_t)f * v] * b[f];
        for (int m = 0; m < o; m++)
            s -= in->ovoo[IDX4(p, x, m, q, v, o, o)] * in->t2[IDX4(r, m, z, y, o, v, v)];
        out[(p * o + q) * o + r] = s;
    }
}

static void raw_v(const Inputs *in, int x, int y, int z, double *out)
{
    const int o = in->o, v = in->v;
    for (int p = 0; p < o; p++)
    for (int q = 0; q < o; q++)
    for (int r = 0; r < o; r++) {
        out[(p * o + q) * o + r] =
            in->ovov[IDX4(p, x, q, y, v, o, v)] * in->t1[(size_t)r * v + z] +
            in->t2[IDX4(q, p, y, x, o, v, v)] * in->fvo[(size_t)z * o + r];
    }
}

/* The six simultaneous (occupied, virtual) permutations.  Permutation t maps
 * a raw tensor r_t computed for virtual ordering VPERM[t] into WW via
 * WW[i,j,k] += r_t[pos_t(i,j,k)], pos_t given by OPERM[t] (ccsd_t.c:99-121,
 * idx0..idx5 used with (a,b,c),(a,c,b),(b,a,c),(b,c,a),(c,a,b),(c,b,a)). */
static const int VPERM[6][3] = {{0,1,2},{0,2,1},{1,0,2},{1,2,0},{2,0,1},{2,1,0}};
/* For WW[i,j,k]: r_t index (P0,P1,P2) where P = (i,j,k)[OPERM[t][.]] */
static const int OPERM[6][3] = {{0,1,2},{0,2,1},{1,0,2},{1,2,0},{2,0,1},{2,1,0}};

static inline int tidx(int o, const int ijk[3], const int *perm)
{
    return (ijk[perm[0]] * o + ijk[perm[1]]) * o + ijk[perm[2]];
}

/* r3(X)[ijk] = 4X[ijk] + X[jki] + X[kij] - 2X[kji] - 2X[ikj] - 2X[jik] */
static void r3(int o, const double *x, double *out)
{
    for (int i = 0; i < o; i++)
    for (int j = 0; j < o; j++)
    for (int k = 0; k < o; k++) {
        out[(i*o+j)*o+k] = 4 * x[(i*o+j)*o+k] + x[(j*o+k)*o+i] + x[(k*o+i)*o+j]
                         - 2 * x[(k*o+j)*o+i] - 2 * x[(i*o+k)*o+j] - 2 * x[(j*o+i)*o+k];
    }
}

static double do_job(const Inputs *in, int a, int b, int c, double ebar, Grads *g,
                     double *buf)
{
    const int o = in->o, v = in->v, n = o + v;
    const size_t ooo = (size_t)o * o * o;
    const int abc[3] = {a, b, c};
    double *w[6], *vv[6];
    for (int t = 0; t < 6; t++) { w[t] = buf + t * ooo; vv[t] = buf + (6 + t) * ooo; }
    double *WW = buf + 12 * ooo, *VV = buf + 13 * ooo, *X = buf + 14 * ooo;
    double *Z = buf + 15 * ooo, *D = buf + 16 * ooo;
    double *Zb = buf + 17 * ooo, *WWb = buf + 18 * ooo, *VVb = buf + 19 * ooo;
    double *tmp = buf + 20 * ooo;

    for (int t = 0; t < 6; t++) {
        raw_w(in, abc[VPERM[t][0]], abc[VPERM[t][1]], abc[VPERM[t][2]], w[t]);
        raw_v(in, abc[VPERM[t][0]], abc[VPERM[t][1]], abc[VPERM[t][2]], vv[t]);
    }
    double fac = (a == c) ? 1.0 / 6 : ((a == b || b == c) ? 0.5 : 1.0);
    double eabc = in->mo_energy[o + a] + in->mo_energy[o + b] + in->mo_energy[o + c];
    for (int i = 0; i < o; i++)
    for (int j = 0; j < o; j++)
    for (int k = 0; k < o; k++) {
        int ijk[3] = {i, j, k};
        size_t m = (size_t)(i * o + j) * o + k;
        double sw = 0, sv = 0;
        for (int t = 0; t < 6; t++) {
            int pos = tidx(o, ijk, OPERM[t]);
            sw += w[t][pos];
            sv += vv[t][pos];
        }
        WW[m] = sw; VV[m] = sv;
        X[m] = sw + 0.5 * sv;
        D[m] = fac / (in->mo_energy[i] + in->mo_energy[j] + in->mo_energy[k] - eabc);
    }
    r3(o, X, Z);
    double e = 0;
    for (size_t m = 0; m < ooo; m++) e += WW[m] * Z[m] * D[m];
    if (!g) return e;

    /* adjoint (ccsd_t_vjp.c:64-117) */
    for (size_t m = 0; m < ooo; m++) {
        Zb[m] = ebar * WW[m] * D[m];
        double db = ebar * WW[m] * Z[m];
        /* mo_energy_bar: d = fac/Delta, dd/dDelta = -d*d/fac */
        int i = (int)(m / ((size_t)o * o)), j = (int)((m / o) % o), k = (int)(m % o);
        double tmpv = db * D[m] * D[m] / fac;
        g->mo_energy_bar[i] -= tmpv; g->mo_energy_bar[j] -= tmpv; g->mo_energy_bar[k] -= tmpv;
        g->mo_energy_bar[o + a] += tmpv; g->mo_energy_bar[o + b] += tmpv; g->mo_energy_bar[o + c] += tmpv;
    }
    r3(o, Zb, tmp);  /* r3 is self-adjoint */
    for (size_t m = 0; m < ooo; m++) {
        WWb[m] = ebar * Z[m] * D[m] + tmp[m];
        VVb[m] = 0.5 * tmp[m];
    }
    (void)n;
    for (int t = 0; t < 6; t++) {
        const int x = abc[VPERM[t][0]], y = abc[VPERM[t][1]], z = abc[VPERM[t][2]];
        /* scatter WWb/VVb back to raw positions of permutation t */
        for (int i = 0; i < o; i++)
        for (int j = 0; j < o; j++)
        for (int k = 0; k < o; k++) {
            int ijk[3] = {i, j, k};
            size_t m = (size_t)(i * o + j) * o + k;
            int pos = tidx(o, ijk, OPERM[t]);
            w[t][pos] = WWb[m];
            vv[t][pos] = VVb[m];
        }
        for (int p = 0; p < o; p++)
        for (int q = 0; q < o; q++)
        for (int r = 0; r < o; r++) {
            double wb = w[t][(p * o + q) * o + r];
            double vb = vv[t][(p * o + q) * o + r];
            for (int f = 0; f < v; f++) {
                g->ovvv_bar[IDX4(p, x, f, y, v, v, v)] += wb * in->t2[IDX4(r, q, z, f, o, v, v)];
                g->t2_bar[IDX4(r, q, z, f, o, v, v)] += wb * in->ovvv[IDX4(p, x, f, y, v, v, v)];
            }
            for (int m = 0; m < o; m++) {
                g->ovoo_bar[IDX4(p, x, m, q, v, o, o)] -= wb * in->t2[IDX4(r, m, z, y, o, v, v)];
                g->t2_bar[IDX4(r, m, z, y, o, v, v)] -= wb * in->ovoo[IDX4(p, x, m, q, v, o, o)];
            }
            g->ovov_bar[IDX4(p, x, q, y, v, o, v)] += vb * in->t1[(size_t)r * v + z];
            g->t1_bar[(size_t)r * v + z] += vb * in->ovov[IDX4(p, x, q, y, v, o, v)];
            g->t2_bar[IDX4(q, p, y, x, o, v, v)] += vb * in->fvo[(size_t)z * o + r];
            g->fvo_bar[(size_t)z * o + r] += vb * in->t2[IDX4(q, p, y, x, o, v, v)];
        }
    }
    return e;
}

static size_t grad_len(int o, int v, int which)
{
    size_t n = (size_t)o + v;
    switch (which) {
    case 0: return n;
    case 1: return (size_t)o * v;
    case 2: return (size_t)o * o * v * v;
    case 3: return (size_t)o * v * o * o;
    case 4: return (size_t)o * v * o * v;
    case 5: return (size_t)o * v * v * v;
    default: return (size_t)v * o;
    }
}

/*
 * Energy (and, when want_grad != 0, the VJP with adjoint seed ybar) over jobs
 * a in [a0,a1), b<=a, c<=b.  Gradients are ACCUMULATED (+=) into the caller's
 * arrays, as the reference's ccsd_t_energy_vjp does (ccsd_t.py:89-106).
 * Returns 0 on success, -1 on bad arguments, -2 on allocation failure.
 */
int triples_oracle_energy_vjp(int nocc, int nvir,
                              const double *mo_energy, const double *t1, const double *t2,
                              const double *ovoo, const double *ovov, const double *ovvv,
                              const double *fvo, double ybar, int want_grad, int a0, int a1,
                              double *e_out,
                              double *mo_energy_bar, double *t1_bar, double *t2_bar,
                              double *ovoo_bar, double *ovov_bar, double *ovvv_bar,
                              double *fvo_bar)
{
    if (nocc <= 0 || nvir <= 0 || a0 < 0 || a1 > nvir || a0 > a1 || !e_out) return -1;
    Inputs in = {nocc, nvir, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo};
    double *outs[7] = {mo_energy_bar, t1_bar, t2_bar, ovoo_bar, ovov_bar, ovvv_bar, fvo_bar};
    const double ebar = 2.0 * ybar;
    size_t njobs = 0;
    for (int a = a0; a < a1; a++) njobs += (size_t)(a + 1) * (a + 2) / 2;
    int *jobs = (int *)malloc(sizeof(int) * 3 * (njobs + 1));
    if (!jobs) return -2;
    size_t m = 0;
    for (int a = a0; a < a1; a++)
        for (int b = 0; b <= a; b++)
            for (int c = 0; c <= b; c++, m++) { jobs[3*m] = a; jobs[3*m+1] = b; jobs[3*m+2] = c; }

    const size_t ooo = (size_t)nocc * nocc * nocc;
    double etot = 0;
    int fail = 0;
#pragma omp parallel reduction(+:etot)
    {
        double *buf = (double *)malloc(sizeof(double) * 21 * ooo);
        Grads gl, *gp = NULL;
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *priv[7] = {0};
        if (want_grad) {
            for (int w = 0; w < 7; w++) {
                if (tid == 0) priv[w] = outs[w];
                else priv[w] = (double *)calloc(grad_len(nocc, nvir, w), sizeof(double));
                if (!priv[w]) {
#pragma omp atomic write
                    fail = 1;
                }
            }
            gl.mo_energy_bar = priv[0]; gl.t1_bar = priv[1]; gl.t2_bar = priv[2];
            gl.ovoo_bar = priv[3]; gl.ovov_bar = priv[4]; gl.ovvv_bar = priv[5];
            gl.fvo_bar = priv[6];
            gp = &gl;
        }
        if (!buf) {
#pragma omp atomic write
            fail = 1;
        }
#pragma omp barrier
        if (!fail) {
#pragma omp for schedule(dynamic)
            for (size_t k = 0; k < njobs; k++)
                etot += do_job(&in, jobs[3*k], jobs[3*k+1], jobs[3*k+2], ebar, gp, buf);
        }
        if (want_grad && tid != 0) {
            for (int w = 0; w < 7; w++) {
                if (!priv[w]) continue;
                size_t len = grad_len(nocc, nvir, w);
#pragma omp critical
                {
                    for (size_t i = 0; i < len; i++) outs[w][i] += priv[w][i];
                }
                free(priv[w]);
            }
        }
        free(buf);
    }
    free(jobs);
    if (fail) return -2;
    *e_out = 2.0 * etot;
    return 0;
}
