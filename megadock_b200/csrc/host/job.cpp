// Job level of the C ABI: one MEGADOCK command line end to end.
//
// md_job_create  = Parameter::initialize + Control::initialize + the host part
//                  of Docking::rec_init (src/parameter.cpp:21-236,
//                  src/control.cpp:18-88, src/docking.cpp:128-191)
// md_job_run     = Control::execute without the detail/CSV outputs:
//                  receptor FFT, every rotation through the device pipeline,
//                  the score merge and the .out file (src/control.cpp:468-529,
//                  src/docking.cpp:194-346, 399-453)
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/md_b200.h"
#include "host.h"

using namespace mdb;

struct md_job {
    Params p;
    Tables tab;
    Molecule rec, lig;
    int ng1 = 0, nf1 = 0;
    std::vector<float> gc, rec_r, rec_i, lig_xyz;
    std::vector<md_pose> poses, top;
    std::string err, log;
};

extern "C" {

int md_rotation_matrix(const float *theta, float *m) {
    if (!theta || !m) return MD_ERR_ARG;
    rotation_matrix(theta, m);
    return MD_OK;
}

int md_sort_poses(md_pose *poses, int n, int nout) {
    if (n < 0 || (n > 0 && !poses)) return MD_ERR_ARG;
    nout = std::max(0, std::min(nout, n));
    // best score first; equal scores keep their input order (one of the orders
    // the reference's unstable partial_sort may produce)
    std::stable_sort(poses, poses + n, [](const md_pose &a, const md_pose &b) { return a.score > b.score; });
    (void)nout;
    return MD_OK;
}

int md_job_create(int argc, const char **argv, md_job **out) {
    if (!out) return MD_ERR_ARG;
    md_job *job = new md_job;
    *out = job;
    std::vector<std::string> store(argv, argv + argc);
    std::vector<char *> av;
    for (auto &s : store) av.push_back(&s[0]);
    av.push_back(nullptr);
    int rc = parse_command_line(argc, av.data(), job->p, job->err, job->log);
    if (rc) return rc;
    if (!load_tables(data_dir(), job->tab, job->err)) return MD_ERR_IO;
    if ((rc = read_molecule(job->p.rec_file, job->tab, job->p.grid_width, job->rec, job->err, job->log))) return rc;
    if ((rc = read_molecule(job->p.lig_file, job->tab, job->p.grid_width, job->lig, job->err, job->log))) return rc;
    if ((rc = size_grids(job->p, job->tab, job->rec, job->lig, job->err, job->log))) return rc;
    // Docking::initialize (src/docking.cpp:18-32)
    job->ng1 = std::max(job->rec.num_grid, job->lig.num_grid);
    job->nf1 = job->ng1 * 2;
    job->gc = grid_coordinates(job->ng1, job->p.grid_width);
    receptor_grids(job->rec, job->p, job->gc, job->ng1, job->rec_r, job->rec_i);
    job->lig_xyz = centred_coordinates(job->lig);
    return MD_OK;
}

const char *md_job_error(const md_job *job) { return job ? job->err.c_str() : "null job"; }

const char *md_job_log(const md_job *job) { return job ? job->log.c_str() : ""; }

void md_job_destroy(md_job *job) { delete job; }

int md_job_run(md_job *job, md_ctx *ctx) {
    if (!job) return MD_ERR_ARG;
    md_ctx *own = nullptr;
    if (!ctx) {
        int rc = md_ctx_create(0, &own);
        if (rc) {
            job->err = "cannot create a device context on device 0";
            return rc;
        }
        ctx = own;
    }
    auto fail = [&](int rc) {
        job->err = md_last_error(ctx);
        if (own) md_ctx_destroy(own);
        return rc;
    };
    int rc;
    if ((rc = md_set_grid(ctx, job->nf1, job->p.grid_width, job->gc.data()))) return fail(rc);
    if ((rc = md_receptor_fft(ctx, job->rec_r.data(), job->rec_i.data()))) return fail(rc);
    if ((rc = md_ligand_data(ctx, job->lig.na(), job->lig_xyz.data(), job->lig.radius.data(),
                             job->lig.charge.data(), job->p.lig_core)))
        return fail(rc);
    const int nrot = job->p.num_rot(), t = job->p.num_sort;
    std::vector<float> rot((size_t)nrot * 9);
    for (int r = 0; r < nrot; ++r) rotation_matrix(&job->p.angles[3 * (size_t)r], &rot[9 * (size_t)r]);
    job->poses.assign((size_t)nrot * t, md_pose{});
    if ((rc = md_dock(ctx, rot.data(), 0, nrot, t, job->poses.data()))) return fail(rc);
    // FFTProcess::sort_index + Docking::output
    job->top = job->poses;
    md_sort_poses(job->top.data(), (int)job->top.size(), job->p.num_output);
    job->top.resize(std::min((size_t)job->p.num_output, job->top.size()));
    std::vector<PoseRec> recs;
    for (const md_pose &q : job->top) recs.push_back(PoseRec{q.score, q.rot, q.i, q.j, q.k});
    if ((rc = write_out_file(job->p.out_file, job->nf1, job->p.grid_width, job->rec, job->lig, job->p, recs,
                             job->err))) {
        if (own) md_ctx_destroy(own);
        return rc;
    }
    if (own) md_ctx_destroy(own);
    return MD_OK;
}

int md_job_dims(const md_job *job, int *ng1, int *nf1, int *na_rec, int *na_lig, int *n_rot, int *t, int *n_out) {
    if (!job) return MD_ERR_ARG;
    if (ng1) *ng1 = job->ng1;
    if (nf1) *nf1 = job->nf1;
    if (na_rec) *na_rec = job->rec.na();
    if (na_lig) *na_lig = job->lig.na();
    if (n_rot) *n_rot = job->p.num_rot();
    if (t) *t = job->p.num_sort;
    if (n_out) *n_out = job->p.num_output;
    return MD_OK;
}

float md_job_grid_width(const md_job *job) { return job ? job->p.grid_width : 0.f; }
float md_job_lig_core(const md_job *job) { return job ? job->p.lig_core : 0.f; }
const char *md_job_out_file(const md_job *job) { return job ? job->p.out_file.c_str() : ""; }

int md_job_grid_coord(const md_job *job, float *out) {
    if (!job || !out) return MD_ERR_ARG;
    std::copy(job->gc.begin(), job->gc.end(), out);
    return MD_OK;
}

int md_job_receptor_grids(const md_job *job, float *r, float *i) {
    if (!job || !r || !i) return MD_ERR_ARG;
    std::copy(job->rec_r.begin(), job->rec_r.end(), r);
    std::copy(job->rec_i.begin(), job->rec_i.end(), i);
    return MD_OK;
}

int md_job_receptor_elec_groups(const md_job *job, const int *group, int ngroups, float *grids) {
    if (!job || !group || ngroups < 1 || !grids) return MD_ERR_ARG;
    receptor_electro(job->rec, job->p, job->gc, job->ng1, job->rec_r, group, ngroups, grids);
    return MD_OK;
}

int md_job_ligand_atoms(const md_job *job, float *xyz, float *radius, float *charge) {
    if (!job) return MD_ERR_ARG;
    if (xyz) std::copy(job->lig_xyz.begin(), job->lig_xyz.end(), xyz);
    if (radius) std::copy(job->lig.radius.begin(), job->lig.radius.end(), radius);
    if (charge) std::copy(job->lig.charge.begin(), job->lig.charge.end(), charge);
    return MD_OK;
}

int md_job_receptor_atoms(const md_job *job, float *xyz, float *radius, float *charge, float *ace) {
    if (!job) return MD_ERR_ARG;
    if (xyz) std::copy(job->rec.xyz.begin(), job->rec.xyz.end(), xyz);
    if (radius) std::copy(job->rec.radius.begin(), job->rec.radius.end(), radius);
    if (charge) std::copy(job->rec.charge.begin(), job->rec.charge.end(), charge);
    if (ace) std::copy(job->rec.ace.begin(), job->rec.ace.end(), ace);
    return MD_OK;
}

int md_job_centers(const md_job *job, float *rc, float *lc) {
    if (!job) return MD_ERR_ARG;
    for (int d = 0; d < 3; ++d) {
        if (rc) rc[d] = job->rec.center[d];
        if (lc) lc[d] = job->lig.center[d];
    }
    return MD_OK;
}

int md_job_rotation_angles(const md_job *job, float *theta) {
    if (!job || !theta) return MD_ERR_ARG;
    std::copy(job->p.angles.begin(), job->p.angles.end(), theta);
    return MD_OK;
}

int md_job_poses(const md_job *job, md_pose *out) {
    if (!job || !out) return MD_ERR_ARG;
    std::copy(job->poses.begin(), job->poses.end(), out);
    return MD_OK;
}

int md_job_top(const md_job *job, md_pose *out) {
    if (!job || !out) return MD_ERR_ARG;
    std::copy(job->top.begin(), job->top.end(), out);
    return MD_OK;
}

}  // extern "C"
