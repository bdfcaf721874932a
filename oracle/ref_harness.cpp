/*
 * Test infrastructure (oracle side only; never linked into the product).
 *
 * A C-ABI harness over the reference's own, unmodified CPU classes, compiled
 * from the reference sources in place (see oracle/Makefile).  It lets tests
 * pin the oracle restatement and the product against the reference itself:
 *   - ref_open:           Control::initialize (src/control.cpp:18-88)
 *   - ref_rec_init:       Docking::rec_init (src/docking.cpp:128-159)
 *   - ref_receptor_grids: receptor rPSC/elec grids left in _Fwork by rec_init
 *   - ref_spectrum:       FFTProcess::_FFT_rec_r/_i (src/fft_process.cpp:294-298)
 *   - ref_ligand_grids:   Docking::ligand_rotationz + create_voxel
 *                         (src/docking.cpp:270-271, 368-396, 162-191)
 *   - ref_dock_rotation:  the CPU per-rotation chain of Docking::dockz
 *                         (src/docking.cpp:262-307) for one rotation
 *   - ref_score_grid:     Re(inverse FFT)/nf3 of the last docked rotation
 * Access to the classes' private members uses the preprocessor only in this
 * translation unit; the reference sources are compiled unmodified.
 */
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <map>
#include <iostream>
#include <fstream>
#include <sstream>
#include <algorithm>
#include <functional>
#include <cassert>
#include <cmath>
#include <unistd.h>
#include <sys/time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define private public
#define protected public
#include "control.h"
#undef private
#undef protected

namespace {
struct Session {
    Parallel *parallel = nullptr;
    CPUTime *cputime = nullptr;
    Control *control = nullptr;
    std::vector<std::string> args;
};
Session *g = nullptr;

Docking *dock() { return g->control->_docking; }
FFTProcess *fftp() { return g->control->_docking->_fft_process; }
}  // namespace

extern "C" {

/* Build the reference's state from a command line (argv[0] is ignored).
 * Returns 0 on success.  The reference calls exit() on bad input. */
int ref_open(int argc, const char **argv) {
    /* a previous session is leaked on purpose: the reference's destructors
     * assume the whole Control::execute sequence ran */
    g = new Session;
    for (int i = 0; i < argc; ++i) g->args.push_back(argv[i]);
    std::vector<char *> av;
    for (auto &s : g->args) av.push_back(const_cast<char *>(s.c_str()));
    av.push_back(nullptr);
    g->cputime = new CPUTime();
    g->cputime->initialize();
    g->parallel = new Parallel(1);
    g->parallel->num_gpu(0);
    g->control = new Control(g->cputime, g->parallel);
    g->control->initialize(argc, av.data());
    return 0;
}

/* ng1, nf1, grid width, ligand and receptor atom counts, rotation count, t. */
int ref_info(int *ng1, int *nf1, float *gw, int *na_lig, int *na_rec, int *nrot, int *t) {
    if (!g) return 1;
    Parameter *p = g->control->_parameter;
    *ng1 = dock()->_Num_grid;
    *nf1 = dock()->_Num_grid * 2;
    *gw = p->grid_width;
    *na_lig = g->control->_ligand->num_atoms();
    *na_rec = g->control->_receptor->num_atoms();
    *nrot = p->_Num_rot_angles;
    *t = p->_Num_sort;
    return 0;
}

int ref_grid_coord(float *out) {
    if (!g) return 1;
    for (int i = 0; i < dock()->_Num_grid; ++i) out[i] = dock()->_Grid_coord[i];
    return 0;
}

int ref_ligand_center(float *c) {
    if (!g) return 1;
    for (int i = 0; i < 3; ++i) c[i] = g->control->_ligand->_Center[i];
    return 0;
}

int ref_receptor_center(float *c) {
    if (!g) return 1;
    for (int i = 0; i < 3; ++i) c[i] = g->control->_receptor->_Center[i];
    return 0;
}

/* Per-atom radius, charge and ACE for the ligand (which=1) or receptor (0). */
int ref_atoms(int which, float *xyz, float *radius, float *charge, float *ace) {
    if (!g) return 1;
    Protein *pr = which ? (Protein *)g->control->_ligand : (Protein *)g->control->_receptor;
    const int na = pr->num_atoms();
    for (int i = 0; i < na; ++i) {
        for (int j = 0; j < 3; ++j) xyz[3 * i + j] = pr->coordinate(i, j);
        radius[i] = pr->_Radius[i];
        charge[i] = pr->_Charge[i];
        ace[i] = pr->_ACE[i];
    }
    return 0;
}

int ref_rec_init(void) {
    if (!g) return 1;
    dock()->rec_init();
    fftp()->top_score_clean();
    return 0;
}

int ref_receptor_grids(float *grid_r, float *grid_i) {
    if (!g) return 1;
    const size_t ng3 = (size_t)dock()->_Num_grid * dock()->_Num_grid * dock()->_Num_grid;
    std::memcpy(grid_r, dock()->_Fwork, sizeof(float) * ng3);
    std::memcpy(grid_i, dock()->_Fwork + ng3, sizeof(float) * ng3);
    return 0;
}

int ref_spectrum(float *re, float *im) {
    if (!g) return 1;
    const size_t nf = (size_t)dock()->_Num_grid * 2;
    const size_t nf3 = nf * nf * nf;
    std::memcpy(re, fftp()->_FFT_rec_r, sizeof(float) * nf3);
    std::memcpy(im, fftp()->_FFT_rec_i, sizeof(float) * nf3);
    return 0;
}

int ref_rotation_angles(int ang, float *theta) {
    if (!g) return 1;
    for (int k = 0; k < 3; ++k) theta[k] = g->control->_parameter->_Zangle[3 * ang + k];
    return 0;
}

/* Rotated, centred ligand coordinates and the rPSC/elec grids for rotation ang. */
int ref_ligand_grids(int ang, float *coord_out, float *grid_r, float *grid_i) {
    if (!g) return 1;
    float theta[3];
    for (int k = 0; k < 3; ++k) theta[k] = g->control->_parameter->_Zangle[3 * ang + k];
    dock()->ligand_rotationz(theta, 0);
    dock()->create_voxel(g->control->_ligand, 0);
    const size_t ng3 = (size_t)dock()->_Num_grid * dock()->_Num_grid * dock()->_Num_grid;
    const int na = g->control->_ligand->num_atoms();
    if (coord_out) std::memcpy(coord_out, dock()->_Mol_coord[0], sizeof(float) * 3 * na);
    if (grid_r) std::memcpy(grid_r, dock()->_Fwork, sizeof(float) * ng3);
    if (grid_i) std::memcpy(grid_i, dock()->_Fwork + ng3, sizeof(float) * ng3);
    return 0;
}

/* The CPU chain of one rotation; writes t records {score, rot, i, j, k}. */
int ref_dock_rotation(int ang, float *score, int *index4) {
    if (!g) return 1;
    float theta[3];
    const int ng1 = dock()->_Num_grid;
    const size_t ng3 = (size_t)ng1 * ng1 * ng1;
    for (int k = 0; k < 3; ++k) theta[k] = g->control->_parameter->_Zangle[3 * ang + k];
    fftp()->rotation_index(0, ang);
    dock()->ligand_rotationz(theta, 0);
    dock()->create_voxel(g->control->_ligand, 0);
    fftp()->ligand_preparation(dock()->_Fwork, dock()->_Fwork + ng3, 0);
    fftp()->fft3d(-1.0, 0);
    fftp()->convolution(0);
    fftp()->fft3d(1.0, 0);
    fftp()->score_sort(0);
    const int t = g->control->_parameter->_Num_sort;
    for (int i = 0; i < t; ++i) {
        score[i] = fftp()->_Top[(size_t)ang * t + i].score;
        for (int k = 0; k < 4; ++k) index4[4 * i + k] = fftp()->_Top[(size_t)ang * t + i].index[k];
    }
    return 0;
}

/* Raw real part of the last inverse FFT (unnormalised), length nf3. */
int ref_score_grid(float *raw) {
    if (!g) return 1;
    const size_t nf = (size_t)dock()->_Num_grid * 2;
    const size_t nf3 = nf * nf * nf;
    for (size_t i = 0; i < nf3; ++i) raw[i] = fftp()->_FFTWout[i][0];
    return 0;
}

/* The merged top-N after ref_dock_rotation over all rotations:
 * FFTProcess::sort_index (src/fft_process.cpp:469-479). */
int ref_sort_index(int nout, float *score, int *index4) {
    if (!g) return 1;
    fftp()->sort_index(nullptr, nullptr);
    for (int r = 0; r < nout; ++r) {
        score[r] = fftp()->top_score(r);
        for (int k = 0; k < 4; ++k) index4[4 * r + k] = fftp()->top_index(r, k);
    }
    return 0;
}

void ref_close(void) {
    /* The reference's destructors assume the full execute() sequence; the
     * session is leaked deliberately (tests open one session per process). */
    g = nullptr;
}

}  // extern "C"
