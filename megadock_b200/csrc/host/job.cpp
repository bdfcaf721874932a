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
#include <array>
#include <cmath>
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
    job->lig_xyz = centred_coordinates(job->lig);
    return MD_OK;
}

// Host receptor grids, built on first use by the accessors that return them
// (the docking path builds them on the device).
static void host_receptor(const md_job *job) {
    md_job *j = const_cast<md_job *>(job);
    if (j->rec_r.empty()) receptor_grids(j->rec, j->p, j->gc, j->ng1, j->rec_r, j->rec_i);
}

const char *md_job_error(const md_job *job) { return job ? job->err.c_str() : "null job"; }

const char *md_job_log(const md_job *job) { return job ? job->log.c_str() : ""; }

void md_job_destroy(md_job *job) { delete job; }

}  // extern "C"

namespace {

// Docking::output_detail (src/docking.cpp:456-898): the .detail and .csv
// files.  Score terms come from md_pose_terms (the reference's summation
// order on the GPU); RMSD, near-native flags and formatting follow the
// reference on the host, including its use of the unrotated ligand
// coordinates in the RMSD (only the translation enters it).
int write_detail(md_job *job, md_ctx *ctx) {
    const Params &p = job->p;
    const int ng1 = job->ng1, nf1 = job->nf1;
    const float gw = p.grid_width;
    // receptor grid without the ACE term (the reference sets the ACE ratio to 0)
    std::vector<float> rpsc((size_t)ng1 * ng1 * ng1);
    {
        const std::vector<float> xyz = centred_coordinates(job->rec);
        int rc = md_receptor_build(ctx, job->rec.na(), xyz.data(), job->rec.radius.data(), job->rec.charge.data(),
                                   job->rec.ace.data(), p.rec_core, 0.0f, p.elec_ratio, 0, rpsc.data(), nullptr);
        if (rc) {
            job->err = md_last_error(ctx);
            return rc;
        }
    }
    float diff[3];
    int cor[3];
    for (int i = 0; i < 3; ++i) {
        diff[i] = job->rec.center[i] - job->lig.center[i];
        cor[i] = (int)std::round(diff[i] / gw);
        if (cor[i] < 0) cor[i] += nf1;
    }
    // poses: 7 around the position that restores the input placement, then the top list
    std::vector<int> tem;
    std::vector<float> rot;
    std::vector<std::array<int, 3>> cors;
    float ident[9];
    const float zero[3] = {0.f, 0.f, 0.f};
    rotation_matrix(zero, ident);
    int c[3] = {cor[0], cor[1], cor[2]};
    for (int rank = 0; rank < 7; ++rank) {
        if (rank == 1) c[0]--;
        if (rank == 2) c[0] += 2;
        if (rank == 3) { c[0]--; c[1]--; }
        if (rank == 4) c[1] += 2;
        if (rank == 5) { c[1]--; c[2]--; }
        if (rank == 6) c[2] += 2;
        cors.push_back({c[0], c[1], c[2]});
        for (int k = 0; k < 3; ++k) tem.push_back((3 * ng1 - c[k]) % (2 * ng1));
        rot.insert(rot.end(), ident, ident + 9);
    }
    for (const md_pose &q : job->top) {
        const int t[3] = {q.i, q.j, q.k};
        cors.push_back({q.i, q.j, q.k});
        for (int k = 0; k < 3; ++k) tem.push_back((3 * ng1 - t[k]) % (2 * ng1));
        float m[9];
        rotation_matrix(&p.angles[3 * (size_t)q.rot], m);
        rot.insert(rot.end(), m, m + 9);
    }
    const int n = (int)cors.size();
    std::vector<float> terms((size_t)n * 9);
    int rc = md_pose_terms(ctx, rpsc.data(), rot.data(), n, tem.data(), terms.data());
    if (rc) {
        job->err = md_last_error(ctx);
        return rc;
    }
    // atom classes: 1 C-alpha, 2 backbone C or N, 0 others (src/protein.cpp:51-60)
    const int na = job->lig.na();
    std::vector<int> type(na);
    int n_ca = 0, n_bb = 0;
    for (int i = 0; i < na; ++i) {
        const std::string &a = job->lig.atom_type[i];
        type[i] = a.compare(0, 3, "CA ") == 0 ? 1 : (a.compare(0, 2, "C ") == 0 || a.compare(0, 2, "N ") == 0) ? 2 : 0;
        n_ca += type[i] == 1;
        n_bb += type[i] > 0;
    }
    auto rmsd_ca = [&](const int *tm) {
        float lca = 0.0f, lbb = 0.0f;
        for (int i = 0; i < na; ++i)
            for (int k = 0; k < 3; ++k) {
                if (type[i] <= 0) continue;
                const float orig = job->lig.xyz[3 * (size_t)i + k];
                const float moved = orig + gw * (tm[k] - ng1) + diff[k];
                const double d2 = std::pow(moved - orig, 2.0);
                if (type[i] == 1) lca = (float)(lca + d2);
                lbb = (float)(lbb + d2);
            }
        (void)lbb;
        return (float)std::sqrt(lca / n_ca);
    };
    FILE *fd = std::fopen(p.out_detail.c_str(), "w");
    if (!fd) {
        job->err = "[ERROR] Output_detail file [" + p.out_detail + "] not open!!";
        return MD_ERR_IO;
    }
    FILE *fc = std::fopen(p.out_csv.c_str(), "w");
    if (!fc) {
        std::fclose(fd);
        job->err = "[ERROR] Output_csv file [" + p.out_csv + "] not open!!";
        return MD_ERR_IO;
    }
    std::fprintf(fd, "%d\t%.2f\n", nf1, gw);
    std::fprintf(fd, "\t%f\t%f\t%f\n", 0.0f, 0.0f, 0.0f);
    std::fprintf(fd, "%s\t%f\t%f\t%f\n", p.rec_file.c_str(), job->rec.center[0], job->rec.center[1],
                 job->rec.center[2]);
    std::fprintf(fd, "%s\t%f\t%f\t%f\n", p.lig_file.c_str(), job->lig.center[0], job->lig.center[1],
                 job->lig.center[2]);
    std::fprintf(fd, "\nElec score ratio: %6.2f\nACE  score ratio: %6.2f\n", p.elec_ratio, p.ace_ratio);
    std::fprintf(fd, "\ncorrect position: angle = (%5.2f,%5.2f,%5.2f), trans = (%3d,%3d,%3d) \n\n", 0.0f, 0.0f,
                 0.0f, cor[0], cor[1], cor[2]);
    std::fprintf(fd, " *** score around correct position *** \n\n");
    const char *cols = "Rank   Angle               Trans         total       rPSC     rPSC(+)  rPSC(-)  ELEC       "
                       "RecACE     LCARMSD NearNat";
    std::fprintf(fd, "%s\n", cols);
    const float nn_thr = 5.0f;
    for (int r = 0; r < 7; ++r) {
        const float *t = &terms[9 * (size_t)r];
        const float total = t[0] + t[1] + t[2];
        const float rm = rmsd_ca(&tem[3 * (size_t)r]);
        std::fprintf(fd, "%5d: (%5.2f,%5.2f,%5.2f) (%3d,%3d,%3d) %11.2f %8.0f %8.0f %8.0f %10.2f %10.2f %7.3f %7d\n",
                     r + 1, 0.0f, 0.0f, 0.0f, cors[r][0], cors[r][1], cors[r][2], total, t[0], t[3], t[4], t[1],
                     t[2], rm, rm < nn_thr ? 1 : 0);
    }
    std::fprintf(fd, "\n *** docking results *** \n\n%s\n", cols);
    std::fprintf(fc, "Rank,Anglex,Angley,Anglez,Transi,Transj,Transk,total,rPSC,rPSC_gain,rPSC_penalty,ELEC ,RecACE,"
                     "LCARMSD,NearNat\n");
    const float pi = (float)(4.0 * std::atan(1.0));
    for (size_t r = 0; r < job->top.size(); ++r) {
        const size_t q = 7 + r;
        const float *t = &terms[9 * q];
        const float s_rpsc = t[3] + t[4], s_elec = t[5] + t[6], s_ace = t[7] + t[8];
        const float total = s_rpsc + s_elec + s_ace;
        float th[3];
        for (int k = 0; k < 3; ++k) {
            th[k] = p.angles[3 * (size_t)job->top[r].rot + k];
            if (th[k] >= pi) th[k] = (float)(th[k] - pi * 2.0);
        }
        const float rm = rmsd_ca(&tem[3 * q]);
        std::fprintf(fd, "%5d: (%5.2f,%5.2f,%5.2f) (%3d,%3d,%3d) %11.2f %8.0f %8.0f %8.0f %10.2f %10.2f %7.3f %7d\n",
                     (int)r + 1, th[0], th[1], th[2], cors[q][0], cors[q][1], cors[q][2], total, s_rpsc, t[3], t[4],
                     s_elec, s_ace, rm, rm < nn_thr ? 1 : 0);
        std::fprintf(fc, "%d, %f,%f,%f,%d,%d,%d,%f,%f,%f,%f,%f,%f,%f,%d\n", (int)r + 1, th[0], th[1], th[2],
                     cors[q][0], cors[q][1], cors[q][2], total, s_rpsc, t[3], t[4], s_elec, s_ace, rm,
                     rm < nn_thr ? 1 : 0);
    }
    const bool ok = std::fclose(fd) == 0;
    if (std::fclose(fc) != 0 || !ok) {
        job->err = "[ERROR] writing the detail output";
        return MD_ERR_IO;
    }
    return MD_OK;
}

}  // namespace

extern "C" {

int md_job_receptor_to(const md_job *job, md_ctx *ctx) {
    if (!job || !ctx) return MD_ERR_ARG;
    const std::vector<float> xyz = centred_coordinates(job->rec);
    return md_receptor_build(ctx, job->rec.na(), xyz.data(), job->rec.radius.data(), job->rec.charge.data(),
                             job->rec.ace.data(), job->p.rec_core, job->p.ace_ratio, job->p.elec_ratio, 1, nullptr,
                             nullptr);
}

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
    if ((rc = md_job_receptor_to(job, ctx))) return fail(rc);   // receptor grids and R^ on the device
    if ((rc = md_ligand_data(ctx, job->lig.na(), job->lig_xyz.data(), job->lig.radius.data(),
                             job->lig.charge.data(), job->p.lig_core)))
        return fail(rc);
    const int nrot = job->p.num_rot(), t = job->p.num_sort;
    std::vector<float> rot((size_t)nrot * 9);
    for (int r = 0; r < nrot; ++r) rotation_matrix(&job->p.angles[3 * (size_t)r], &rot[9 * (size_t)r]);
    std::vector<md_pose> poses((size_t)nrot * t, md_pose{});
    if ((rc = md_dock(ctx, rot.data(), 0, nrot, t, poses.data()))) return fail(rc);
    rc = md_job_write_out(job, ctx, poses.data(), (int)poses.size());
    if (own) md_ctx_destroy(own);
    return rc;
}

int md_job_write_out(md_job *job, md_ctx *ctx, const md_pose *poses, int n) {
    if (!job || (n > 0 && !poses) || n != job->p.num_rot() * job->p.num_sort) {
        if (job) job->err = "md_job_write_out needs n_rot * t poses";
        return MD_ERR_ARG;
    }
    job->poses.assign(poses, poses + n);
    // FFTProcess::sort_index + Docking::output
    job->top = job->poses;
    md_sort_poses(job->top.data(), (int)job->top.size(), job->p.num_output);
    job->top.resize(std::min((size_t)job->p.num_output, job->top.size()));
    int rc;
    if (job->p.detail_output && ctx && (rc = write_detail(job, ctx))) return rc;
    std::vector<PoseRec> recs;
    for (const md_pose &q : job->top) recs.push_back(PoseRec{q.score, q.rot, q.i, q.j, q.k});
    return write_out_file(job->p.out_file, job->nf1, job->p.grid_width, job->rec, job->lig, job->p, recs, job->err);
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
    host_receptor(job);
    std::copy(job->rec_r.begin(), job->rec_r.end(), r);
    std::copy(job->rec_i.begin(), job->rec_i.end(), i);
    return MD_OK;
}

int md_job_receptor_elec_groups(const md_job *job, const int *group, int ngroups, float *grids) {
    if (!job || !group || ngroups < 1 || !grids) return MD_ERR_ARG;
    host_receptor(job);
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
