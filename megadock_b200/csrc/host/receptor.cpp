// Receptor grids, once per receptor-ligand pair (host side).
//
// Real part: rPSC core (value -a, default -45) for cells within sqrt(1.5) R of
// an atom, cavities closed by ray casting from the six faces plus two in-place
// 6-neighbour propagation sweeps (the sweeps are order dependent, so they run
// in the same sequential order), then for every non-core cell the sum over
// atoms within (R + 3.6) A of 1 + ACE * (-0.8) * d_ace  (src/receptor.cpp:20-254).
// Imaginary part: sum over charged atoms of e * beta * q / (eps(r) * r) with
// beta = -2800 and the distance-dependent dielectric 4 / 38r-224 / 80 for
// r <= 6 / 6 < r < 8 / r >= 8, skipping core cells (src/receptor.cpp:258-346).
// Mixed float/double expressions keep the reference's promotions.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "host.h"

namespace mdb {

void receptor_grids(const Molecule &rec, const Params &p, const std::vector<float> &gc, int ng1,
                    std::vector<float> &grid_r, std::vector<float> &grid_i) {
    const int ng2 = ng1 * ng1;
    const size_t ng3 = (size_t)ng2 * ng1;
    const int na = rec.na();
    const float gw = p.grid_width;
    const float epsilon = p.rec_core;
    const float open_space = -7777.0f;
    const std::vector<float> xyz = centred_coordinates(rec);

    grid_r.assign(ng3, 0.0f);
    grid_i.assign(ng3, 0.0f);
    std::vector<float> shell(ng3, 0.0f);

    // squared per-axis distances atom -> grid centre
    std::vector<float> dx((size_t)na * ng1), dy((size_t)na * ng1), dz((size_t)na * ng1);
    for (int l = 0; l < na; ++l)
        for (int g = 0; g < ng1; ++g) {
            float a = xyz[3 * l] - gc[g], b = xyz[3 * l + 1] - gc[g], c = xyz[3 * l + 2] - gc[g];
            dx[(size_t)l * ng1 + g] = a * a;
            dy[(size_t)l * ng1 + g] = b * b;
            dz[(size_t)l * ng1 + g] = c * c;
        }
    auto origin = [&](float c) { return (int)(c / gw + ng1 / 2); };

    // core cells
    {
        const int reach = (int)((2.4 + gw - 0.01) / gw);
        for (int l = 0; l < na; ++l) {
            const float r = rec.radius[l];
            const float core2 = r * r * 1.5f;
            const int i0 = origin(xyz[3 * l]), j0 = origin(xyz[3 * l + 1]), k0 = origin(xyz[3 * l + 2]);
            const float *ax = &dx[(size_t)l * ng1], *ay = &dy[(size_t)l * ng1], *az = &dz[(size_t)l * ng1];
            for (int i = std::max(i0 - reach, 0); i < std::min(i0 + reach + 1, ng1); ++i)
                for (int j = std::max(j0 - reach, 0); j < std::min(j0 + reach + 1, ng1); ++j)
                    for (int k = std::max(k0 - reach, 0); k < std::min(k0 + reach + 1, ng1); ++k)
                        if (ax[i] + ay[j] + az[k] < core2) grid_r[(size_t)ng2 * i + ng1 * j + k] = epsilon;
        }
    }

    // open space reachable in a straight line from a face (order independent)
    for (int a = 0; a < ng1; ++a)
        for (int b = 0; b < ng1; ++b) {
            const size_t base[3] = {(size_t)a + (size_t)ng1 * b, (size_t)b * ng2 + (size_t)a * ng1,
                                    (size_t)a * ng2 + b};
            const size_t step[3] = {(size_t)ng2, 1, (size_t)ng1};
            for (int ax = 0; ax < 3; ++ax) {
                for (int k = 0; k < ng1; ++k) {
                    float &v = grid_r[base[ax] + step[ax] * k];
                    if (v == epsilon) break;
                    v = open_space;
                }
                for (int k = ng1 - 1; k >= 0; --k) {
                    float &v = grid_r[base[ax] + step[ax] * k];
                    if (v == epsilon) break;
                    v = open_space;
                }
            }
        }

    // two in-place propagation sweeps (sequential order matters)
    for (int sweep = 0; sweep < 2; ++sweep) {
        for (size_t c = ng2; c < ng3 - ng2; ++c) {
            const int j = (int)((c / ng1) % ng1);
            if (j < 2 || j > ng1 - 2) continue;
            const int k = (int)(c % ng1);
            if (k < 2 || k > ng1 - 2) continue;
            if (grid_r[c] != open_space) continue;
            const size_t nb[6] = {c + 1, c - 1, c + ng1, c - ng1, c + ng2, c - ng2};
            for (size_t n : nb)
                if (grid_r[n] == 0) grid_r[n] = open_space;
        }
    }
    for (size_t c = 0; c < ng3; ++c)
        if (grid_r[c] == 0) grid_r[c] = epsilon;   // closed cavities become core
    for (size_t c = 0; c < ng3; ++c)
        if (grid_r[c] == open_space) grid_r[c] = 0;

    // surface shell: rPSC count + ACE term
    {
        const int reach = (int)((12 + gw - 0.01) / gw);
        for (int l = 0; l < na; ++l) {
            const float rd = rec.radius[l] + 3.6f;
            const float shell2 = rd * rd;
            const double term = 1.0 + rec.ace[l] * (-0.8) * p.ace_ratio;
            const int i0 = origin(xyz[3 * l]), j0 = origin(xyz[3 * l + 1]), k0 = origin(xyz[3 * l + 2]);
            const float *ax = &dx[(size_t)l * ng1], *ay = &dy[(size_t)l * ng1], *az = &dz[(size_t)l * ng1];
            for (int i = std::max(i0 - reach, 0); i < std::min(i0 + reach + 1, ng1); ++i) {
                if (ax[i] > shell2) continue;
                for (int j = std::max(j0 - reach, 0); j < std::min(j0 + reach + 1, ng1); ++j) {
                    if (ax[i] + ay[j] > shell2) continue;
                    for (int k = std::max(k0 - reach, 0); k < std::min(k0 + reach + 1, ng1); ++k) {
                        if (ax[i] + ay[j] + az[k] < shell2) {
                            float &v = shell[(size_t)ng2 * i + ng1 * j + k];
                            v = (float)(v + term);
                        }
                    }
                }
            }
        }
    }
    for (size_t c = 0; c < ng3; ++c)
        if (grid_r[c] != epsilon) grid_r[c] = shell[c];

    receptor_electro(rec, p, gc, ng1, grid_r, nullptr, 1, grid_i.data());
}

void receptor_electro(const Molecule &rec, const Params &p, const std::vector<float> &gc, int ng1,
                      const std::vector<float> &grid_r, const int *group, int ngroups, float *out) {
    const int ng2 = ng1 * ng1;
    const size_t ng3 = (size_t)ng2 * ng1;
    const int na = rec.na();
    const std::vector<float> xyz = centred_coordinates(rec);
    std::fill(out, out + ng3 * ngroups, 0.0f);
    std::vector<float> dx(ng1), dy(ng1), dz(ng1);
    const float beta = -2800.0f;
    const float e_ratio = p.elec_ratio;
    const float width = gc[1] - gc[0];
    const float charge_per_grid = -1 * width * 80.0f / (beta * e_ratio);
    auto origin_w = [&](float c) { return (int)(c / width + ng1 / 2); };
    for (int l = 0; l < na; ++l) {
        const float q = rec.charge[l];
        const float aq = std::fabs(q);
        if (aq <= 1.0e-6f) continue;
        const int g = group ? group[l] : 0;
        if (g < 0 || g >= ngroups) continue;
        float *grid_i = out + ng3 * g;
        int reach;
        if (aq < 0.07) reach = 4;
        else if (aq < 0.21) reach = 5;
        else reach = (int)(aq / charge_per_grid);
        for (int c = 0; c < ng1; ++c) {
            float a = xyz[3 * l] - gc[c], b = xyz[3 * l + 1] - gc[c], d = xyz[3 * l + 2] - gc[c];
            dx[c] = a * a;
            dy[c] = b * b;
            dz[c] = d * d;
        }
        const int i0 = origin_w(xyz[3 * l]), j0 = origin_w(xyz[3 * l + 1]), k0 = origin_w(xyz[3 * l + 2]);
        for (int i = std::max(i0 - reach, 0); i < std::min(i0 + reach + 1, ng1); ++i)
            for (int j = std::max(j0 - reach, 0); j < std::min(j0 + reach + 1, ng1); ++j) {
                const float d2 = dx[i] + dy[j];
                for (int k = std::max(k0 - reach, 0); k < std::min(k0 + reach + 1, ng1); ++k) {
                    const size_t c = (size_t)ng2 * i + ng1 * j + k;
                    if (grid_r[c] < 0.0) continue;   // receptor core
                    const float r = std::sqrt(d2 + dz[k]);
                    float eps;
                    if (r >= 8.0f) eps = 80.0f;
                    else if (r > 6.0f) eps = 38.0f * r + -224.0f;
                    else eps = 4.0f;
                    grid_i[c] += e_ratio * beta * q / eps / r;
                }
            }
    }
}

}  // namespace mdb
