/*
 * Test infrastructure (oracle side only; never linked into the product).
 *
 * Plain-C restatement of MEGADOCK's per-rotation docking steps, written from
 * the reference's behaviour.  It is the checker for the device pipeline; its
 * own correctness is pinned by tests against the reference compiled from its
 * sources (oracle/_ref, tests/test_oracle.py).  Float semantics: every step is
 * the reference's float expression in the same association order, compiled
 * with -ffp-contract=off.
 *
 *   oracle_rotation_matrix  src/docking.cpp:376-384
 *   oracle_rotate           src/docking.cpp:386-393
 *   oracle_ligand_grids     src/ligand.cpp:20-198 (rPSC), :200-239 (charges),
 *                           :241-260 (radii), src/protein.cpp:134-165 (distances)
 *   oracle_score_sort       src/fft_process.cpp:399-458
 */
#include "md_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

void oracle_rotation_matrix(const float *th, float *m) {
    const float c0 = cosf(th[0]), s0 = sinf(th[0]);
    const float c1 = cosf(th[1]), s1 = sinf(th[1]);
    const float c2 = cosf(th[2]), s2 = sinf(th[2]);
    m[0] = c0 * c2 - s0 * c1 * s2;
    m[1] = -c0 * s2 - s0 * c1 * c2;
    m[2] = s0 * s1;
    m[3] = s0 * c2 + c0 * c1 * s2;
    m[4] = -s0 * s2 + c0 * c1 * c2;
    m[5] = -c0 * s1;
    m[6] = s1 * s2;
    m[7] = s1 * c2;
    m[8] = c1;
}

void oracle_rotate(int na, const float *xyz, const float *m, float *out) {
    for (int l = 0; l < na; ++l) {
        const float x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        for (int d = 0; d < 3; ++d) out[3 * l + d] = m[3 * d] * x + m[3 * d + 1] * y + m[3 * d + 2] * z;
    }
}

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

/* Mark cells within r2 of each atom (search box +-2 around the atom's cell). */
static void fill_spheres(int na, const float *xr, const float *r2, int ng, float gw, const float *dx,
                         const float *dy, const float *dz, float *grid, float value, float skip_value,
                         int use_skip) {
    const int ng2 = ng * ng;
    for (int l = 0; l < na; ++l) {
        const int ci = (int)(xr[3 * l] / gw + ng / 2);
        const int cj = (int)(xr[3 * l + 1] / gw + ng / 2);
        const int ck = (int)(xr[3 * l + 2] / gw + ng / 2);
        const float *ax = dx + (size_t)l * ng, *ay = dy + (size_t)l * ng, *az = dz + (size_t)l * ng;
        for (int i = imax(ci - 2, 0); i < imin(ci + 3, ng); ++i)
            for (int j = imax(cj - 2, 0); j < imin(cj + 3, ng); ++j) {
                const float d2 = ax[i] + ay[j];
                for (int k = imax(ck - 2, 0); k < imin(ck + 3, ng); ++k) {
                    float *cell = &grid[(size_t)ng2 * i + (size_t)ng * j + k];
                    if (use_skip && *cell == skip_value) continue;
                    if (d2 + az[k] < r2[l]) *cell = value;
                }
            }
    }
}

/* Interior cells equal to `from` with a zero 6-neighbour become `to`. */
static void mark_boundary(float *g, int ng, float from, float to) {
    const int ng2 = ng * ng;
    for (int i = 1; i < ng - 1; ++i)
        for (int j = 1; j < ng - 1; ++j)
            for (int k = 1; k < ng - 1; ++k) {
                const size_t c = (size_t)ng2 * i + (size_t)ng * j + k;
                if (g[c] != from) continue;
                if (g[c - 1] == 0 || g[c + 1] == 0 || g[c - ng] == 0 || g[c + ng] == 0 || g[c - ng2] == 0 ||
                    g[c + ng2] == 0)
                    g[c] = to;
            }
}

void oracle_ligand_grids(int na, const float *xr, const float *radius, const float *charge, int ng, float gw,
                         const float *gc, float delta, float *grid_r, float *grid_i) {
    const size_t ng3 = (size_t)ng * ng * ng;
    const int ng2 = ng * ng;
    float *dx = malloc(sizeof(float) * (size_t)na * ng);
    float *dy = malloc(sizeof(float) * (size_t)na * ng);
    float *dz = malloc(sizeof(float) * (size_t)na * ng);
    float *core2 = malloc(sizeof(float) * (size_t)na);
    float *surf2 = malloc(sizeof(float) * (size_t)na);
    for (int l = 0; l < na; ++l) {
        core2[l] = radius[l] * radius[l] * 1.5f;
        surf2[l] = radius[l] * radius[l] * 1.0f;
        for (int g = 0; g < ng; ++g) {
            float a = xr[3 * l] - gc[g], b = xr[3 * l + 1] - gc[g], c = xr[3 * l + 2] - gc[g];
            dx[(size_t)l * ng + g] = a * a;
            dy[(size_t)l * ng + g] = b * b;
            dz[(size_t)l * ng + g] = c * c;
        }
    }
    memset(grid_r, 0, sizeof(float) * ng3);
    memset(grid_i, 0, sizeof(float) * ng3);
    const float swollen = -8888.0f;
    /* core spheres */
    fill_spheres(na, xr, core2, ng, gw, dx, dy, dz, grid_r, delta, 0.f, 0);
    /* scrape the swollen surface: interior core cells touching empty space */
    mark_boundary(grid_r, ng, delta, swollen);
    for (size_t c = (size_t)ng2; c < ng3 - ng2; ++c)
        if (grid_r[c] == swollen) grid_r[c] = 0.0f;
    /* surface spheres on non-core cells */
    fill_spheres(na, xr, surf2, ng, gw, dx, dy, dz, grid_r, 1.0f, delta, 1);
    /* with a core value other than the surface value, core cells next to
     * empty space become surface */
    if (delta != 1.0f) mark_boundary(grid_r, ng, delta, 1.0f);
    /* charges at the clamped nearest cell, in atom order */
    const float pad = ng * gw / 2;
    for (int l = 0; l < na; ++l) {
        const int i = imax(0, imin(ng - 1, (int)((xr[3 * l] + pad) / gw)));
        const int j = imax(0, imin(ng - 1, (int)((xr[3 * l + 1] + pad) / gw)));
        const int k = imax(0, imin(ng - 1, (int)((xr[3 * l + 2] + pad) / gw)));
        grid_i[(size_t)i * ng2 + (size_t)j * ng + k] += charge[l];
    }
    free(dx);
    free(dy);
    free(dz);
    free(core2);
    free(surf2);
}

void oracle_score_sort(const float *raw, int nf, int t, float *scores, int *index3) {
    const long long nf2 = (long long)nf * nf, nf3 = nf2 * nf;
    if (t == 1) {
        /* running maximum from 0.0 with strict '<': first index wins ties,
         * all-non-positive grids give (0, index 0) */
        float best = 0.0f;
        long long bi = 0;
        for (long long i = 0; i < nf3; ++i)
            if (best < raw[i]) {
                best = raw[i];
                bi = i;
            }
        scores[0] = best / (float)nf3;
        index3[0] = (int)(bi / nf2);
        index3[1] = (int)((bi / nf) % nf);
        index3[2] = (int)(bi % nf);
        return;
    }
    /* insertion top-t with strict '>' from a -99999 sentinel */
    float *s = malloc(sizeof(float) * t);
    long long *ix = malloc(sizeof(long long) * t);
    for (int q = 0; q < t; ++q) {
        s[q] = -99999.0f;
        ix[q] = 0;
    }
    for (long long i = 0; i < nf3; ++i) {
        const float v = raw[i] / (float)nf3;
        if (v < s[t - 1]) continue;
        for (int q = 0; q < t; ++q) {
            if (v > s[q]) {
                for (int r = t - 1; r > q; --r) {
                    s[r] = s[r - 1];
                    ix[r] = ix[r - 1];
                }
                s[q] = v;
                ix[q] = i;
                break;
            }
        }
    }
    for (int q = 0; q < t; ++q) {
        scores[q] = s[q];
        index3[3 * q] = (int)(ix[q] / nf2);
        index3[3 * q + 1] = (int)((ix[q] / nf) % nf);
        index3[3 * q + 2] = (int)(ix[q] % nf);
    }
    free(s);
    free(ix);
}
