/* CPU oracle: a plain-C restatement of the reference's 2-body/3-body path.
 *
 * TEST INFRASTRUCTURE ONLY.  The tests, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py use this as the checker; the product never links
 * it.  It is pinned against the reference itself (oracle/_ref, built from the
 * reference sources by oracle/build_ref.py) and against the reference's golden
 * vectors in tests/.
 *
 * Everything is FP64.  The file must be compiled with -ffp-contract=off so
 * that the n-mer search reproduces the reference's x86-64 arithmetic (no FMA
 * contraction) operation by operation.
 *
 * Functions and the reference code they restate:
 *   mbxo_invert_box      InvertUnitCell            tools/math_tools.cpp:37-64
 *   mbxo_fix_monomers    FixMonomerCoordinates     bblock/sys_tools.cpp:257-320
 *   mbxo_close_image     GetCloseDimerImage        bblock/sys_tools.cpp:322-366
 *   mbxo_add_clusters    AddClusters (n_max 2, 3)  bblock/sys_tools.cpp:472-592
 *                        + XyzToCloud              kdtree/kdtree_utils.h:196-278
 *                        + GetFractionalCoordinates kdtree/kdtree_utils.h:165-190
 *                        + radius search predicate kdtree/nanoflann.hpp:166-167
 *   mbxo_pip_eval        the generated PIPs, from their expanded term tables
 *   mbxo_holder_eval     the evaluator classes (x2b_v9x, x3b_v2x, the MB-nrg
 *                        CH4 classes), driven by the declarative description
 *                        in mbx_b200/specs.py
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---------------------------------------------------------------- boxes */

int mbxo_invert_box(const double *b, double *inv) {
    double det = b[0] * (b[4] * b[8] - b[7] * b[5]) - b[1] * (b[3] * b[8] - b[5] * b[6]) +
                 b[2] * (b[3] * b[7] - b[4] * b[6]);
    if (fabs(det) < 1e-36) return 1;
    double di = 1 / det;
    inv[0] = (b[4] * b[8] - b[7] * b[5]) * di;
    inv[1] = (b[2] * b[7] - b[1] * b[8]) * di;
    inv[2] = (b[1] * b[5] - b[2] * b[4]) * di;
    inv[3] = (b[5] * b[6] - b[3] * b[8]) * di;
    inv[4] = (b[0] * b[8] - b[2] * b[6]) * di;
    inv[5] = (b[3] * b[2] - b[0] * b[5]) * di;
    inv[6] = (b[3] * b[7] - b[6] * b[4]) * di;
    inv[7] = (b[6] * b[1] - b[0] * b[7]) * di;
    inv[8] = (b[0] * b[4] - b[3] * b[1]) * di;
    return 0;
}

static void to_frac(const double *inv, const double *p, double *f) {
    f[0] = inv[0] * p[0] + inv[3] * p[1] + inv[6] * p[2];
    f[1] = inv[1] * p[0] + inv[4] * p[1] + inv[7] * p[2];
    f[2] = inv[2] * p[0] + inv[5] * p[1] + inv[8] * p[2];
}

static void to_cart(const double *b, const double *f, double *p) {
    p[0] = b[0] * f[0] + b[3] * f[1] + b[6] * f[2];
    p[1] = b[1] * f[0] + b[4] * f[1] + b[7] * f[2];
    p[2] = b[2] * f[0] + b[5] * f[1] + b[8] * f[2];
}

void mbxo_fix_monomers(int nmon, const long *first_index, const int *nat, const double *box, const double *inv,
                       double *xyz) {
    for (int i = 0; i < nmon; ++i) {
        double *p = xyz + 3 * first_index[i];
        double f0[3], f[3];
        to_frac(inv, p, f0);
        f0[0] -= floor(f0[0] + 0.5);
        f0[1] -= floor(f0[1] + 0.5);
        f0[2] -= floor(f0[2] + 0.5);
        to_cart(box, f0, p);
        for (int j = 1; j < nat[i]; ++j) {
            double *q = p + 3 * j;
            to_frac(inv, q, f);
            f[0] -= floor(f[0] - f0[0] + 0.5);
            f[1] -= floor(f[1] - f0[1] + 0.5);
            f[2] -= floor(f[2] - f0[2] + 0.5);
            to_cart(box, f, q);
        }
    }
}

/* Moves monomer 2 (nat2 atoms) to the image closest to monomer 1, judged on
 * the first atoms in fractional coordinates. */
void mbxo_close_image(const double *box, const double *inv, const double *xyz1, int nat2, double *xyz2) {
    double f1[3], f2[3], f[3], d[3];
    to_frac(inv, xyz1, f1);
    to_frac(inv, xyz2, f2);
    d[0] = floor(f2[0] - f1[0] + 0.5);
    d[1] = floor(f2[1] - f1[1] + 0.5);
    d[2] = floor(f2[2] - f1[2] + 0.5);
    for (int j = 0; j < nat2; ++j) {
        to_frac(inv, xyz2 + 3 * j, f);
        f[0] -= d[0];
        f[1] -= d[1];
        f[2] -= d[2];
        to_cart(box, f, xyz2 + 3 * j);
    }
}

/* ------------------------------------------------------------ n-mer search */

static void frac_coords(const double *box, const double *pt, double *c) {
    double A = box[0];
    double B = sqrt(box[3] * box[3] + box[4] * box[4]);
    double C = sqrt(box[6] * box[6] + box[7] * box[7] + box[8] * box[8]);
    double AdotB = box[0] * box[3];
    double AdotC = box[0] * box[6];
    double BdotC = box[3] * box[6] + box[4] * box[7];
    double gamma = acos(AdotB / A / B);
    double beta = acos(AdotC / A / C);
    double alpha = acos(BdotC / B / C);
    double ca = cos(alpha), cb = cos(beta), cg = cos(gamma), sg = sin(gamma);
    double omega = A * B * C * sqrt(1 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg);
    c[0] = 1 / A * pt[0] - cg / A / sg * pt[1] + B * C * (ca * cg - cb) / omega / sg * pt[2];
    c[1] = 1 / B / sg * pt[1] + A * C * (cb * cg - ca) / omega / sg * pt[2];
    c[2] = A * B * sg / omega * pt[2];
}

typedef struct {
    double x, y, z;
} pt3;

/* The point cloud of the reference: wrapped first-atom positions, and with
 * PBC seven periodic copies of every point at index i + s*np (s = 1..7). */
static pt3 *make_cloud(int np, const double *xyz, int use_pbc, const double *box, const double *inv) {
    size_t size = (size_t)np * (use_pbc ? 8 : 1);
    pt3 *pts = (pt3 *)calloc(size, sizeof(pt3));
    static const int indxs[3] = {0, -1, 1};
    for (int i = 0; i < np; ++i) {
        double p[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
        double uvw[3] = {0, 0, 0};
        if (use_pbc) {
            double f[3];
            to_frac(inv, p, f);
            f[0] -= floor(f[0] + 0.5);
            f[1] -= floor(f[1] + 0.5);
            f[2] -= floor(f[2] + 0.5);
            to_cart(box, f, p);
            frac_coords(box, p, uvw);
        }
        pts[i].x = p[0];
        pts[i].y = p[1];
        pts[i].z = p[2];
        if (!use_pbc) continue;
        for (int m2 = 0; m2 < 3; ++m2) {
            int m = indxs[m2];
            if ((uvw[0] + m) > 1.0 || (uvw[0] + m) < -1.0) continue;
            for (int n2 = 0; n2 < 3; ++n2) {
                int n = indxs[n2];
                if ((uvw[1] + n) > 1.0 || (uvw[1] + n) < -1.0) continue;
                for (int l2 = 0; l2 < 3; ++l2) {
                    if (m2 == 0 && n2 == 0 && l2 == 0) continue;
                    int l = indxs[l2];
                    if ((uvw[2] + l) > 1.0 || (uvw[2] + l) < -1.0) continue;
                    int shift;
                    if (m == 0 && n == 0)
                        shift = 1;
                    else if (m == 0 && l == 0)
                        shift = 2;
                    else if (n == 0 && l == 0)
                        shift = 3;
                    else if (m != 0 && n != 0 && l != 0)
                        shift = 4;
                    else if (m == 0)
                        shift = 5;
                    else if (n == 0)
                        shift = 6;
                    else
                        shift = 7;
                    double sx = (double)m * box[0] + (double)n * box[3] + (double)l * box[6];
                    double sy = (double)m * box[1] + (double)n * box[4] + (double)l * box[7];
                    double sz = (double)m * box[2] + (double)n * box[5] + (double)l * box[8];
                    size_t at = (size_t)i + (size_t)shift * np;
                    pts[at].x = p[0] + sx;
                    pts[at].y = p[1] + sy;
                    pts[at].z = p[2] + sz;
                }
            }
        }
    }
    return pts;
}

typedef struct {
    long idx;
    double d;
} match;

static int cmp_match(const void *a, const void *b) {
    const match *x = (const match *)a, *y = (const match *)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->idx < y->idx) ? -1 : (x->idx > y->idx);
}

/* Dimers (nmax 2) or trimers (nmax 3) in the reference's monomer indices.
 * mon_xyz: first-atom positions of the nmon monomers (3 doubles each);
 * tag: the first atom's tag per monomer; is_local per monomer.
 * Writes at most cap n-mers (nmax indices each) into out and returns the
 * total number of n-mers found; counts are exact even when cap is exceeded. */
long mbxo_add_clusters(int nmax, double cutoff, int nmon, int use_pbc, const double *box, const double *inv,
                       const double *mon_xyz, const long *tag, const int *is_local, int use_ghost, long *out,
                       long cap) {
    int *mon_index = (int *)malloc(sizeof(int) * (nmon + 1));
    long *tag_index = (long *)malloc(sizeof(long) * (nmon + 1));
    double *xyz = (double *)malloc(sizeof(double) * 3 * (nmon + 1));
    int np = 0;
    for (int i = 0; i < nmon; ++i) {
        if (use_ghost || is_local[i]) {
            xyz[3 * np] = mon_xyz[3 * i];
            xyz[3 * np + 1] = mon_xyz[3 * i + 1];
            xyz[3 * np + 2] = mon_xyz[3 * i + 2];
            mon_index[np] = i;
            tag_index[np] = tag[i];
            ++np;
        }
    }
    long count = 0;
    if (np < 2 || (nmax > 2 && np < 3)) goto done;
    {
        pt3 *pts = make_cloud(np, xyz, use_pbc, box, inv);
        long npts = (long)np * (use_pbc ? 8 : 1);
        double rc2 = cutoff * cutoff;
        match *mt = (match *)malloc(sizeof(match) * npts);
        for (int i = 0; i < np; ++i) {
            if (!is_local[mon_index[i]]) continue;
            double q[3] = {pts[i].x, pts[i].y, pts[i].z};
            long nm = 0;
            for (long p = 0; p < npts; ++p) {
                double d0 = q[0] - pts[p].x;
                double d1 = q[1] - pts[p].y;
                double d2 = q[2] - pts[p].z;
                double d = d0 * d0 + d1 * d1 + d2 * d2;
                if (d < rc2) {
                    mt[nm].idx = p;
                    mt[nm].d = d;
                    ++nm;
                }
            }
            qsort(mt, nm, sizeof(match), cmp_match);
            if (nmax == 2) {
                for (long j = 0; j < nm; ++j) {
                    long idj = mt[j].idx % np;
                    if (tag_index[i] < tag_index[idj]) {
                        if (count < cap) {
                            out[2 * count] = mon_index[i];
                            out[2 * count + 1] = mon_index[idj];
                        }
                        ++count;
                    }
                }
            } else {
                for (long j = 0; j < nm; ++j) {
                    for (long k = j + 1; k < nm; ++k) {
                        const pt3 *pj = pts + mt[j].idx, *pk = pts + mt[k].idx;
                        double djk0 = pj->x - pk->x, djk1 = pj->y - pk->y, djk2 = pj->z - pk->z;
                        long idj = mt[j].idx % np, idk = mt[k].idx % np;
                        if (idj == i || idk == i || idj == idk) continue;
                        if (djk0 * djk0 + djk1 * djk1 + djk2 * djk2 > rc2 ||
                            (tag_index[i] < tag_index[idj] && tag_index[i] < tag_index[idk])) {
                            if (count < cap) {
                                out[3 * count] = mon_index[i];
                                out[3 * count + 1] = mon_index[idj];
                                out[3 * count + 2] = mon_index[idk];
                            }
                            ++count;
                        }
                    }
                }
            }
        }
        free(mt);
        free(pts);
    }
done:
    free(mon_index);
    free(tag_index);
    free(xyz);
    return count;
}

/* ---------------------------------------------------------------- the PIP */

/* P(a, x) = sum_t a[k_t] * c_t * prod_{i < deg_t} x[v_t,i]; g (optional) gets
 * dP/dx (overwritten).  tv: tw variable slots per term (tw >= the degree). */
double mbxo_pip_eval(int nvars, long nterms, const int *tk, const double *tc, const int *tdeg, const int *tv,
                     int tw, const double *a, const double *x, double *g) {
    double e = 0.0;
    if (g)
        for (int j = 0; j < nvars; ++j) g[j] = 0.0;
    for (long t = 0; t < nterms; ++t) {
        const int *v = tv + (long)tw * t;
        int deg = tdeg[t];
        double c = a[tk[t]] * tc[t];
        double m = c;
        for (int i = 0; i < deg; ++i) m *= x[v[i]];
        e += m;
        if (g) {
            for (int i = 0; i < deg; ++i) {
                double d = c;
                for (int j = 0; j < deg; ++j)
                    if (j != i) d *= x[v[j]];
                g[v[i]] += d;
            }
        }
    }
    return e;
}

/* ------------------------------------------------------------ evaluators */

/* Switch of the N2O5 - H2O - H2O 3b on S = s12 + s13 + s23
 * (mbnrg_3b_A1B2C4_D1E2_D1E2_deg3_v1.cpp:2464-2471, gradient :2563-2570):
 * 0 for S < 1, 1 for S > 2, 1 - cos^2((S - 1) pi / 2) between; *dS (optional)
 * gets dsw/dS = -(pi / 2) sin(pi S) strictly inside (1, 2), else 0. */
static double switch_cos2(double S, double *dS) {
    if (dS) *dS = (S > 1.0 && S < 2.0) ? -(M_PI / 2.0) * sin(M_PI * S) : 0.0;
    if (S < 1.0) return 0.0;
    if (S > 2.0) return 1.0;
    double c = cos((S - 1.0) * M_PI / 2.0);
    return 1.0 - c * c;
}

#define MBXO_MAXV 128  /* polynomial variables of one evaluator, at most */

typedef struct {
    int nbody;
    int nreal;      /* real atoms across the n-mer, holder order */
    int nsites;     /* nreal + virtual sites */
    int nat[3];     /* atoms per monomer */
    int nlp;        /* lone-pair pairs */
    int lp[3][4];   /* (monomer, first real site, X+ site, X- site) */
    int nvars;
    int vkind[MBXO_MAXV];  /* 0 exp, 1 coul */
    int vs1[MBXO_MAXV], vs2[MBXO_MAXV];
    double vk[MBXO_MAXV], vd[MBXO_MAXV];
    int sw_triple;  /* 0 pair, 1 triple, 2 triple minus 2 s0 s1 s2, 3 1 - cos^2((S - 1) pi / 2), S = s0+s1+s2 */
    double ri, rf;
    int skip;       /* 0 pair_gt, 1 two_of_three_gt, 2 all_three_gt */
    double gin, gout;
    int virial_raw; /* 1: virial over the unswitched polynomial gradient
                       (x2b_A1B2C4_D1E2_deg3_v1x.cpp:1353-1391) */
} mbxo_spec;

static double f_switch(double r, double ri, double rf, double *g) {
    if (r > rf) {
        *g = 0.0;
        return 0.0;
    } else if (r > ri) {
        double t1 = M_PI / (rf - ri);
        double x = (r - ri) * t1;
        *g = -sin(x) * t1 / 2.0;
        return (1.0 + cos(x)) / 2.0;
    }
    *g = 0.0;
    return 1.0;
}

static void lp_setup(const double *ohh, double gin, double gout, double *x1, double *x2, double *oh1, double *oh2) {
    for (int i = 0; i < 3; ++i) {
        oh1[i] = ohh[i + 3] - ohh[i];
        oh2[i] = ohh[i + 6] - ohh[i];
    }
    double v[3] = {oh1[1] * oh2[2] - oh1[2] * oh2[1], oh1[2] * oh2[0] - oh1[0] * oh2[2],
                   oh1[0] * oh2[1] - oh1[1] * oh2[0]};
    for (int i = 0; i < 3; ++i) {
        double in_plane = ohh[i] + 0.5 * gin * (oh1[i] + oh2[i]);
        double out_of_plane = gout * v[i];
        x1[i] = in_plane + out_of_plane;
        x2[i] = in_plane - out_of_plane;
    }
}

static void lp_grads(const double *g1, const double *g2, double gin, double gout, const double *oh1,
                     const double *oh2, double *grd) {
    double gm[3] = {g1[0] - g2[0], g1[1] - g2[1], g1[2] - g2[2]};
    double t1[3] = {oh2[1] * gm[2] - oh2[2] * gm[1], oh2[2] * gm[0] - oh2[0] * gm[2], oh2[0] * gm[1] - oh2[1] * gm[0]};
    double t2[3] = {oh1[1] * gm[2] - oh1[2] * gm[1], oh1[2] * gm[0] - oh1[0] * gm[2], oh1[0] * gm[1] - oh1[1] * gm[0]};
    for (int i = 0; i < 3; ++i) {
        double gsum = g1[i] + g2[i];
        double in_plane = 0.5 * gin * gsum;
        double gh1 = in_plane + gout * t1[i];
        double gh2 = in_plane - gout * t2[i];
        grd[i + 0] += gsum - (gh1 + gh2);
        grd[i + 3] += gh1;
        grd[i + 6] += gh2;
    }
}

/* Evaluates n n-mers.  xyz: n * nreal * 3 doubles, holder order, already
 * imaged; grad (optional): same layout, accumulated (+=); virial (optional,
 * 9): accumulated; e_out (optional, n): switched energy per n-mer.
 * Returns the summed switched energy. */
double mbxo_holder_eval(const mbxo_spec *s, long nterms, const int *tk, const double *tc, const int *tdeg,
                        const int *tv, int tw, const double *a, long n, const double *xyz, double *grad,
                        double *virial, double *e_out) {
    double etot = 0.0;
    double vir[6] = {0, 0, 0, 0, 0, 0};
    int first[3];
    first[0] = 0;
    for (int m = 1; m < s->nbody; ++m) first[m] = first[m - 1] + s->nat[m - 1];
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : etot, vir[:6])
    for (long t = 0; t < n; ++t) {
        const double *w = xyz + (size_t)t * s->nreal * 3;
        double r[3], d[3][3];
        int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        int npair = s->nbody == 2 ? 1 : 3;
        for (int p = 0; p < npair; ++p) {
            const double *a1 = w + 3 * first[pairs[p][0]], *a2 = w + 3 * first[pairs[p][1]];
            for (int c = 0; c < 3; ++c) d[p][c] = a1[c] - a2[c];
            r[p] = sqrt(d[p][0] * d[p][0] + d[p][1] * d[p][1] + d[p][2] * d[p][2]);
        }
        int skip;
        if (s->skip == 0)
            skip = r[0] > s->rf;
        else if (s->skip == 1)
            skip = (r[0] > s->rf && r[1] > s->rf) || (r[0] > s->rf && r[2] > s->rf) || (r[1] > s->rf && r[2] > s->rf);
        else
            skip = r[0] > s->rf && r[1] > s->rf && r[2] > s->rf;
        if (skip) {
            if (e_out) e_out[t] = 0.0;
            continue;
        }
        double sites[32][3];
        double oh1[3][3], oh2[3][3];
        for (int i = 0; i < s->nreal; ++i)
            for (int c = 0; c < 3; ++c) sites[i][c] = w[3 * i + c];
        for (int l = 0; l < s->nlp; ++l)
            lp_setup(sites[s->lp[l][1]], s->gin, s->gout, sites[s->lp[l][2]], sites[s->lp[l][3]], oh1[l], oh2[l]);
        double x[MBXO_MAXV], gx[MBXO_MAXV], dv[MBXO_MAXV][3];
        for (int v = 0; v < s->nvars; ++v) {
            const double *p1 = sites[s->vs1[v]], *p2 = sites[s->vs2[v]];
            double g0 = p1[0] - p2[0], g1 = p1[1] - p2[1], g2 = p1[2] - p2[2];
            double rr = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
            double e1 = exp(s->vk[v] * (s->vd[v] - rr));
            double gg;
            if (s->vkind[v] == 0) {
                x[v] = e1;
                gg = -s->vk[v] * e1 / rr;
            } else {
                double rinv = 1.0 / rr;
                x[v] = e1 * rinv;
                gg = -(s->vk[v] + rinv) * x[v] * rinv;
            }
            dv[v][0] = g0 * gg;
            dv[v][1] = g1 * gg;
            dv[v][2] = g2 * gg;
        }
        double ep = mbxo_pip_eval(s->nvars, nterms, tk, tc, tdeg, tv, tw, a, x, grad ? gx : NULL);
        double sw, gsw[3];
        double sp[3], gp[3];
        if (!s->sw_triple) {
            sp[0] = f_switch(r[0], s->ri, s->rf, &gp[0]);
            sw = sp[0];
        } else {
            for (int p = 0; p < 3; ++p) sp[p] = f_switch(r[p], s->ri, s->rf, &gp[p]);
            sw = sp[0] * sp[1] + sp[0] * sp[2] + sp[1] * sp[2];
            if (s->sw_triple == 2) sw -= 2.0 * sp[0] * sp[1] * sp[2];
            if (s->sw_triple == 3) sw = switch_cos2(sp[0] + sp[1] + sp[2], NULL);
        }
        double es = sw * ep;
        etot += es;
        if (e_out) e_out[t] = es;
        if (!grad) continue;
        double sg[32][3];
        memset(sg, 0, sizeof(sg));
        for (int v = 0; v < s->nvars; ++v) {
            for (int c = 0; c < 3; ++c) {
                double dd = gx[v] * dv[v][c];
                sg[s->vs1[v]][c] += dd;
                sg[s->vs2[v]][c] -= dd;
            }
        }
        for (int l = 0; l < s->nlp; ++l)
            lp_grads(sg[s->lp[l][2]], sg[s->lp[l][3]], s->gin, s->gout, oh1[l], oh2[l], sg[s->lp[l][1]]);
        double *gout = grad + (size_t)t * s->nreal * 3;
        double tg[32][3];
        for (int i = 0; i < s->nreal; ++i)
            for (int c = 0; c < 3; ++c) tg[i][c] = sw * sg[i][c];
        if (!s->sw_triple) {
            gsw[0] = gp[0] * ep / r[0];
            for (int c = 0; c < 3; ++c) {
                double dd = gsw[0] * d[0][c];
                tg[first[0]][c] += dd;
                tg[first[1]][c] -= dd;
            }
        } else {
            double c2 = s->sw_triple == 2 ? 2.0 : 0.0;
            if (s->sw_triple == 3) {
                double dS;
                switch_cos2(sp[0] + sp[1] + sp[2], &dS);
                for (int p = 0; p < 3; ++p) gsw[p] = gp[p] * dS * ep / r[p];
            } else {
                gsw[0] = gp[0] * (sp[1] + sp[2] - c2 * sp[1] * sp[2]) * ep / r[0];
                gsw[1] = gp[1] * (sp[0] + sp[2] - c2 * sp[0] * sp[2]) * ep / r[1];
                gsw[2] = gp[2] * (sp[0] + sp[1] - c2 * sp[0] * sp[1]) * ep / r[2];
            }
            for (int c = 0; c < 3; ++c) {
                tg[first[0]][c] += gsw[0] * d[0][c] + gsw[1] * d[1][c];
                tg[first[1]][c] += gsw[2] * d[2][c] - gsw[0] * d[0][c];
                tg[first[2]][c] -= gsw[1] * d[1][c] + gsw[2] * d[2][c];
            }
        }
        for (int i = 0; i < s->nreal; ++i)
            for (int c = 0; c < 3; ++c) gout[3 * i + c] += tg[i][c];
        for (int i = 0; i < s->nreal; ++i) {
            const double *q = w + 3 * i;
            const double *vg = s->virial_raw ? sg[i] : tg[i];
            vir[0] -= q[0] * vg[0];
            vir[1] -= q[0] * vg[1];
            vir[2] -= q[0] * vg[2];
            vir[3] -= q[1] * vg[1];
            vir[4] -= q[1] * vg[2];
            vir[5] -= q[2] * vg[2];
        }
    }
    /* the reference fills the lower triangle from the upper one
       (x2b-v9x.cpp:1786-1788, x3b-v2x.cpp:1724-1726) */
    if (virial) {
        virial[0] += vir[0];
        virial[1] += vir[1];
        virial[2] += vir[2];
        virial[4] += vir[3];
        virial[5] += vir[4];
        virial[8] += vir[5];
        virial[3] = virial[1];
        virial[6] = virial[2];
        virial[7] = virial[5];
    }
    return etot;
}

/* Design-matrix row: dE/da_k for one n-mer = sw * p_k(x) (the gradient of
 * the switched energy with respect to the linear coefficients).  out: ncoef
 * doubles (overwritten).  Returns 0 when the n-mer is skipped (row zero). */
int mbxo_holder_dcoef(const mbxo_spec *s, int ncoef, long nterms, const int *tk, const double *tc, const int *tdeg,
                      const int *tv, int tw, const double *xyz, double *out) {
    for (int k = 0; k < ncoef; ++k) out[k] = 0.0;
    int first[3];
    first[0] = 0;
    for (int m = 1; m < s->nbody; ++m) first[m] = first[m - 1] + s->nat[m - 1];
    const double *w = xyz;
    double r[3];
    int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    int npair = s->nbody == 2 ? 1 : 3;
    for (int p = 0; p < npair; ++p) {
        const double *a1 = w + 3 * first[pairs[p][0]], *a2 = w + 3 * first[pairs[p][1]];
        double d0 = a1[0] - a2[0], d1 = a1[1] - a2[1], d2 = a1[2] - a2[2];
        r[p] = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    }
    int skip;
    if (s->skip == 0)
        skip = r[0] > s->rf;
    else if (s->skip == 1)
        skip = (r[0] > s->rf && r[1] > s->rf) || (r[0] > s->rf && r[2] > s->rf) || (r[1] > s->rf && r[2] > s->rf);
    else
        skip = r[0] > s->rf && r[1] > s->rf && r[2] > s->rf;
    if (skip) return 0;
    double sites[32][3], oh1[3][3], oh2[3][3], x[MBXO_MAXV];
    for (int i = 0; i < s->nreal; ++i)
        for (int c = 0; c < 3; ++c) sites[i][c] = w[3 * i + c];
    for (int l = 0; l < s->nlp; ++l)
        lp_setup(sites[s->lp[l][1]], s->gin, s->gout, sites[s->lp[l][2]], sites[s->lp[l][3]], oh1[l], oh2[l]);
    for (int v = 0; v < s->nvars; ++v) {
        const double *p1 = sites[s->vs1[v]], *p2 = sites[s->vs2[v]];
        double g0 = p1[0] - p2[0], g1 = p1[1] - p2[1], g2 = p1[2] - p2[2];
        double rr = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
        double e1 = exp(s->vk[v] * (s->vd[v] - rr));
        x[v] = s->vkind[v] == 0 ? e1 : e1 / rr;
    }
    double sp[3], gp[3], sw;
    if (!s->sw_triple) {
        sw = f_switch(r[0], s->ri, s->rf, &gp[0]);
    } else {
        for (int p = 0; p < 3; ++p) sp[p] = f_switch(r[p], s->ri, s->rf, &gp[p]);
        sw = sp[0] * sp[1] + sp[0] * sp[2] + sp[1] * sp[2];
        if (s->sw_triple == 2) sw -= 2.0 * sp[0] * sp[1] * sp[2];
        if (s->sw_triple == 3) sw = switch_cos2(sp[0] + sp[1] + sp[2], NULL);
    }
    for (long t = 0; t < nterms; ++t) {
        double m = tc[t];
        for (int i = 0; i < tdeg[t]; ++i) m *= x[tv[(long)tw * t + i]];
        out[tk[t]] += m;
    }
    for (int k = 0; k < ncoef; ++k) out[k] *= sw;
    return 1;
}

/* The polynomial variables of every n-mer (the first half of holder_eval:
 * skip rule, lone-pair sites, x_v = exp(k (d0 - r)) [/ r]); x_out[n][nvars],
 * live[t] = 0 for an n-mer beyond the evaluator's cutoff (its x left 0). */
long mbxo_holder_vars(const mbxo_spec *s, long n, const double *xyz, double *x_out, unsigned char *live) {
    int first[3];
    long nlive = 0;
    first[0] = 0;
    for (int m = 1; m < s->nbody; ++m) first[m] = first[m - 1] + s->nat[m - 1];
#pragma omp parallel for schedule(static) reduction(+ : nlive)
    for (long t = 0; t < n; ++t) {
        const double *w = xyz + (size_t)t * s->nreal * 3;
        double *x = x_out + (size_t)t * s->nvars;
        double r[3];
        int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        int npair = s->nbody == 2 ? 1 : 3;
        for (int p = 0; p < npair; ++p) {
            const double *a1 = w + 3 * first[pairs[p][0]], *a2 = w + 3 * first[pairs[p][1]];
            double d0 = a1[0] - a2[0], d1 = a1[1] - a2[1], d2 = a1[2] - a2[2];
            r[p] = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        }
        int skip;
        if (s->skip == 0)
            skip = r[0] > s->rf;
        else if (s->skip == 1)
            skip = (r[0] > s->rf && r[1] > s->rf) || (r[0] > s->rf && r[2] > s->rf) || (r[1] > s->rf && r[2] > s->rf);
        else
            skip = r[0] > s->rf && r[1] > s->rf && r[2] > s->rf;
        for (int v = 0; v < s->nvars; ++v) x[v] = 0.0;
        live[t] = !skip;
        if (skip) continue;
        ++nlive;
        double sites[32][3], oh1[3][3], oh2[3][3];
        for (int i = 0; i < s->nreal; ++i)
            for (int c = 0; c < 3; ++c) sites[i][c] = w[3 * i + c];
        for (int l = 0; l < s->nlp; ++l)
            lp_setup(sites[s->lp[l][1]], s->gin, s->gout, sites[s->lp[l][2]], sites[s->lp[l][3]], oh1[l], oh2[l]);
        for (int v = 0; v < s->nvars; ++v) {
            const double *p1 = sites[s->vs1[v]], *p2 = sites[s->vs2[v]];
            double g0 = p1[0] - p2[0], g1 = p1[1] - p2[1], g2 = p1[2] - p2[2];
            double rr = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
            double e1 = exp(s->vk[v] * (s->vd[v] - rr));
            x[v] = s->vkind[v] == 0 ? e1 : e1 / rr;
        }
    }
    return nlive;
}

long mbxo_spec_size(void) { return (long)sizeof(mbxo_spec); }
