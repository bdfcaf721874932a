/*
 * megadock-b200: C ABI of the B200-native per-rotation FFT docking path.
 *
 * The reference (akiyamalab/MEGADOCK) has no plugin API: its seam is the C++
 * class FFTProcess (src/fft_process.h:168-195), called by Docking
 * (src/docking.cpp).  Each entry point below states which FFTProcess /
 * Docking / Control member it replaces.  Conventions:
 *   - every function returns an int status, MD_OK (0) on success; nothing
 *     calls exit() (the reference calls exit(1) on every error);
 *   - md_last_error(ctx) (or md_job_error(job)) describes the last failure;
 *   - host buffers are caller-owned; device buffers are owned by the context;
 *   - one context per device, not shared between threads without a lock;
 *   - all work is stream-ordered on the context's stream (md_set_stream).
 */
#ifndef MD_B200_H
#define MD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    MD_OK = 0,
    MD_ERR_ARG = 1,     /* bad argument (size, pointer, flag) */
    MD_ERR_CUDA = 2,    /* CUDA runtime failure */
    MD_ERR_STATE = 3,   /* call out of order (e.g. dock before receptor) */
    MD_ERR_SIZE = 4,    /* FFT size / atom count beyond what is built */
    MD_ERR_IO = 5,      /* file read/write failure */
    MD_ERR_USAGE = 6    /* command-line usage error */
};

typedef struct md_ctx md_ctx;
typedef struct md_job md_job;

/* One docking pose.  Mirrors SortScore {float score; int index[4]}
 * (src/fft_process.h:40-43): rot = index[0] (rotation number),
 * i/j/k = index[1..3] (translation cell of the FFT grid). */
typedef struct md_pose {
    float score;
    int rot, i, j, k;
} md_pose;

/* ------------------------------------------------------------ device context */

/* Replaces the per-GPU set-up of FFTProcess::alloc_fft (src/fft_process.cpp:79-209)
 * and main()'s device selection (src/main.cpp:75-110). */
int md_ctx_create(int device, md_ctx **out);
void md_ctx_destroy(md_ctx *ctx);               /* FFTProcess::fft_memory_free (:814-875) */
const char *md_last_error(const md_ctx *ctx);
/* Run all work on this cudaStream_t (NULL = the context's own stream). */
int md_set_stream(md_ctx *ctx, void *cuda_stream);
/* 1 when FFT edge nf1 has a built kernel set, else 0. */
int md_fft_size_supported(int nf1);

/* FFTProcess::alloc_array(num_fft) (src/fft_process.cpp:29-76) plus the grid
 * centre coordinates of Docking::rec_init (src/docking.cpp:139-142).
 * nf1 = 2 * ng1; grid_coord has ng1 entries. */
int md_set_grid(md_ctx *ctx, int nf1, float grid_width, const float *grid_coord);

/* FFTProcess::receptor_fft(grid_r, grid_i) (src/fft_process.cpp:212-303):
 * embed the ng1^3 receptor grids at offset ng1/2 and take the forward 3D FFT
 * on the device; the spectrum stays resident. */
int md_receptor_fft(md_ctx *ctx, const float *grid_r, const float *grid_i);
/* Copy the resident receptor spectrum (nf1^3 each, [x][y][z] order) back. */
int md_receptor_spectrum(md_ctx *ctx, float *re, float *im);

/* FFTProcess::ligand_data_transfer_gpu(grid_coord) (src/fft_process.cpp:769-807):
 * centred atom coordinates (3*na), CHARMM radii and charges, and the ligand core
 * value (-b, Ligand::rpscace's delta).  Core/surface radii are R*R*1.5 and
 * R*R*1.0 as in Ligand::precalc (src/ligand.cpp:241-260). */
int md_ligand_data(md_ctx *ctx, int na, const float *xyz_centred, const float *radius, const float *charge,
                   float lig_core);

/* Rotations per launch for md_dock (1 = the plain per-rotation pipeline;
 * > 1 = the batched form, launched as one captured CUDA graph). */
int md_set_batch(md_ctx *ctx, int rotations_per_launch);
/* Free the context's rotation work buffers and captured graphs (receptor,
 * ligand and settings stay); the next docking call allocates them again for
 * its launch shape.  The autotuner calls it after trying large launch groups. */
int md_release_work(md_ctx *ctx);
/* Radix plan of the plane top-t (inverse plane) kernel: 0 the line plans,
 * 1 the kz split reversed, 2 the ky split reversed (t <= 4; larger t uses 0).
 * The autotuner (megadock_b200.tune) picks it together with the batch. */
int md_set_plan(md_ctx *ctx, int plan);
/* Tile shape of the x-line kernel: 8, 16 or 32 kz lines per CTA (default
 * 32); also picked by the autotuner.  Above FFT edge 450 a 32-line tile no
 * longer fits a CTA's shared memory and 16-line tiles run for it. */
int md_set_tile(md_ctx *ctx, int lines);
/* Launch groups of the batched form in flight at once: 2 (default) alternates
 * them over two work sets and two streams so that one group's kernels overlap
 * the next one's; 1 runs them back to back on one stream.  Which is faster
 * depends on the size; the autotuner picks it. */
int md_set_lanes(md_ctx *ctx, int lanes);

/* FFTProcess::cuda_fft (src/fft_process.cpp:502-656) over rotations
 * [first_rot, first_rot + n_rot): rotate, voxelize, FFT, conj(R^) product,
 * inverse FFT, top-t.  rotmat holds 9 floats per rotation (row-major, from
 * md_rotation_matrix).  out receives n_rot * t poses, rotation-major, each
 * rotation's poses best first (the _Top layout, src/fft_process.cpp:640-643).
 * Host buffers; copies are included. */
int md_dock(md_ctx *ctx, const float *rotmat, int first_rot, int n_rot, int t, md_pose *out);
/* Same with device-resident rotation matrices and device output buffer. */
int md_dock_device(md_ctx *ctx, const float *d_rotmat, int first_rot, int n_rot, int t, md_pose *d_out);

/* Batched form over many receptor-ligand pairs of uneven FFT sizes: the
 * reference docks one pair per process and farms pairs out over MPI
 * (src/mpidp.cpp:281-551); here every pair's rotations run in one captured
 * CUDA graph on `runner`'s stream and work buffers.  pairs[p] is a context
 * prepared for pair p (md_set_grid, md_receptor_fft, md_ligand_data, and its
 * rotations per launch from md_set_batch) on the runner's device;
 * d_rotmat[p] holds 9 * n_rot[p] floats and d_out[p] receives n_rot[p] * t
 * poses (device buffers).  Rotation numbers in the poses count from 0 per
 * pair.  Asynchronous on the runner's stream. */
int md_dock_pairs(md_ctx *runner, md_ctx *const *pairs, int npairs, const float *const *d_rotmat, const int *n_rot,
                  int t, md_pose *const *d_out);

/* Per-stage device time of md_dock_device's launches (no graph): stage_ms[5]
 * receives the summed CUDA-event time of the voxelizer (rotation, rPSC classes
 * and ordered charge sums), the forward-plane kernel (y/z FFT), the x-line
 * product kernel, the inverse-plane top-t kernel and the merge kernel;
 * *launches the number of kernel launches.  Replaces the reference's
 * gettimeofday buckets (src/cpu_time.h:35-61). */
int md_dock_profile(md_ctx *ctx, const float *d_rotmat, int first_rot, int n_rot, int t, md_pose *d_out,
                    float *stage_ms, int *launches);

/* Receptor::rpscace + Receptor::electro (src/receptor.cpp:20-346) on the
 * device: the rPSC/ACE real grid and the electrostatic grid of na receptor
 * atoms (coordinates centred on the receptor, radius, charge and ACE value
 * per atom; -a, -d and -e values), bit-exact with the reference's CPU code
 * for grids up to ng1 = 256 (every size the docking kernels are built for).
 * make_receptor = 1 also makes them this
 * context's receptor (R^ for md_dock, and the grids for the adjoint), as
 * md_receptor_fft would; grid_r / grid_i (ng1^3 host floats, may be NULL)
 * receive a copy.  Needs md_set_grid. */
int md_receptor_build(md_ctx *ctx, int na, const float *xyz_centred, const float *radius, const float *charge,
                      const float *ace, float rec_core, float ace_ratio, float elec_ratio, int make_receptor,
                      float *grid_r, float *grid_i);

/* Adjoint (no counterpart in the reference, whose scores are not
 * differentiated): gradient of the smooth loss
 *     L = T * log(sum_r exp(s_r / T))
 * over the per-rotation top-1 scores s_r of the rotations in rotmat
 * (9 * n_rot floats) whose poses top1[n_rot] came from md_dock with t = 1.
 * Outputs (host buffers, any may be NULL): *loss; dL/d(receptor grid) real and
 * imaginary parts d_rec_r/d_rec_i (ng1^3 each, the grids given to
 * md_receptor_fft); dL/d(ligand atom charge) d_charge (na); dL/d(alpha)
 * d_alpha, alpha being the electrostatic weight -e that scales the receptor's
 * imaginary grid (its support held fixed); and, for the n_lig_rot rotations
 * listed in lig_rot (indices into rotmat), dL/d(ligand grid) d_lig_r/d_lig_i
 * (n_lig_rot * ng1^3 each).  Rotations whose top score was clamped to 0 carry
 * no gradient.  FP32 accumulation in a fixed order. */
int md_adjoint_lse(md_ctx *ctx, const float *rotmat, int n_rot, const md_pose *top1, float temperature, float alpha,
                   double *loss, float *d_rec_r, float *d_rec_i, float *d_charge, double *d_alpha,
                   const int *lig_rot, int n_lig_rot, float *d_lig_r, float *d_lig_i);

/* General form of the adjoint: dL/d(parameters) for a loss whose gradient
 * with respect to the scores of n poses is dl_ds[n] (host floats).  Pose p
 * has the rotation rotmat[9p..9p+8] and the translation (i, j, k) of
 * poses[p] (the score and rot fields are not read).  Outputs as for
 * md_adjoint_lse; lig_pose[n_lig] lists poses (indices into the n) whose
 * ligand-grid gradient is wanted.  md_adjoint_lse is this with
 * dl_ds = softmax(s / T). */
int md_adjoint_poses(md_ctx *ctx, const float *rotmat, int n, const md_pose *poses, const float *dl_ds,
                     float *d_rec_r, float *d_rec_i, float *d_charge, const int *lig_pose, int n_lig,
                     float *d_lig_r, float *d_lig_i);

/* Scores of given poses (rotation rotmat[9p..], translation poses[p].i/j/k)
 * formed directly as sum_x Rr(x) Lr(x + t) + Ri(x) Li(x + t): the value of the
 * score grid at that translation (FP32, fixed summation order). */
int md_pose_scores(md_ctx *ctx, const float *rotmat, int n, const md_pose *poses, float *scores);

/* Score terms for the detail output (Docking::output_detail,
 * src/docking.cpp:456-898): for n poses (rotation rotmat[9p..], offsets
 * tem3[3p..] = (3 ng1 - t) mod 2 ng1 of the translation t per axis), nine
 * floats each in terms[9p..]: the direct sums of the rPSC, electrostatic and
 * ACE products, then rPSC+, rPSC-, ELEC+, ELEC-, ACE+, ACE-.  rec_rpsc is the
 * receptor's real grid without the ACE term (ng1^3, host); the real grid
 * with it and the electrostatic grid are those given to md_receptor_fft.
 * Sums in the reference's cell order, no FMA: the reference's floats.  Grids
 * up to ng1 = 256 (every built FFT size); larger ones return MD_ERR_SIZE. */
int md_pose_terms(md_ctx *ctx, const float *rec_rpsc, const float *rotmat, int n, const int *tem3, float *terms);

/* Ligand::rpscace + Ligand::electro (src/ligand.cpp:20-239) of one rotation,
 * computed by the device voxelizer; grid_r/grid_i receive ng1^3 floats. */
int md_ligand_voxels(md_ctx *ctx, const float *rotmat9, float *grid_r, float *grid_i);

/* Allocation-free variant of md_dock_device.  No counterpart in the reference.
 * For callers that cannot allocate device memory (a host framework whose pool
 * allocator owns all device memory, a plugin that must not grow its host's
 * footprint, a loop where cudaMalloc/cudaFree and their device-wide
 * synchronisation are not allowed): every intermediate lives in one 32 MiB
 * file-scope device array that each device loading the library holds until
 * exit.  The caller passes all inputs and outputs as device pointers:
 * grid_coord (ng1), receptor_spectrum (nf1^3 complex as interleaved float
 * pairs re, im; md_receptor_spectrum returns separate re and im arrays, which
 * the caller interleaves), centred xyz (3*na), radius and charge (na),
 * rotmat (9*n_rot), out (n_rot*t poses).  Limits: nf1 <= 128 with a built
 * kernel set, na <= 32768, t <= 64 (else MD_ERR_SIZE); rotations run one per
 * pipeline on `stream` (a cudaStream_t, NULL = default).  The first call on a
 * device does the set-up with that device current: make it before any stream
 * capture.  Every call looks the scratch address up again and repeats the
 * set-up when it changed (after cudaDeviceReset, or in another driver
 * context on that device).  All calls share the one scratch array: calls that overlap on the
 * GPU race, so the caller must serialise them.  Nothing is allocated, freed or
 * synchronised; the call returns once the work is enqueued. */
int md_dock_noalloc(int nf1, float grid_width, const float *d_grid_coord, const float *d_receptor_spectrum, int na,
                    const float *d_xyz_centred, const float *d_radius, const float *d_charge, float lig_core,
                    const float *d_rotmat, int first_rot, int n_rot, int t, md_pose *d_out, void *stream);

/* ------------------------------------------------------------ host helpers */

/* Rotation matrix of Docking::ligand_rotationz (src/docking.cpp:368-396) for
 * ZXZ Euler angles theta[3]; m is row-major. */
int md_rotation_matrix(const float *theta, float *m);

/* FFTProcess::sort_index (src/fft_process.cpp:469-479): order poses by score,
 * best first, for the first nout records (ties keep input order). */
int md_sort_poses(md_pose *poses, int n, int nout);

/* ------------------------------------------------------------ job (CLI) level */

/* Parameter::initialize + Control::initialize (src/parameter.cpp:21-236,
 * src/control.cpp:18-88): parse a MEGADOCK command line (argv[0] ignored),
 * read the PDB files and tables, size the grid, build the receptor grids. */
int md_job_create(int argc, const char **argv, md_job **out);
const char *md_job_error(const md_job *job);
/* Progress and warning text collected while the job was set up. */
const char *md_job_log(const md_job *job);
void md_job_destroy(md_job *job);
/* Control::execute (src/control.cpp:468-529): dock every rotation on ctx and
 * write the .out file.  ctx may be NULL (a context on device 0 is made). */
int md_job_run(md_job *job, md_ctx *ctx);
/* The job's receptor grids built on the device (md_receptor_build with the
 * job's atoms and -a/-d/-e values) and made ctx's receptor; ctx must have the
 * job's grid (md_set_grid with nf1, grid width and grid coordinates). */
int md_job_receptor_to(const md_job *job, md_ctx *ctx);
/* The output half of md_job_run for poses docked elsewhere (for example
 * gathered from several GPUs): the n = n_rot * t poses in rotation-major
 * order are merged (FFTProcess::sort_index, src/fft_process.cpp:469-479) and
 * written as the .out (Docking::output, src/docking.cpp:399-453); with -O and
 * a context the .detail/.csv files too. */
int md_job_write_out(md_job *job, md_ctx *ctx, const md_pose *poses, int n);

/* Job properties (valid after md_job_create). */
int md_job_dims(const md_job *job, int *ng1, int *nf1, int *na_rec, int *na_lig, int *n_rot, int *t,
                int *n_out);
float md_job_grid_width(const md_job *job);
const char *md_job_out_file(const md_job *job);
int md_job_grid_coord(const md_job *job, float *out);                 /* ng1 */
int md_job_receptor_grids(const md_job *job, float *grid_r, float *grid_i); /* ng1^3 */
int md_job_ligand_atoms(const md_job *job, float *xyz_centred, float *radius, float *charge);
int md_job_receptor_atoms(const md_job *job, float *xyz, float *radius, float *charge, float *ace);
/* Table mode (-tb), replacing the MPI job farm of src/mpidp.cpp:132-251,
 * :300-551, :786-914 with a one-process queue on one GPU.  argv is the whole
 * command line (-tb <table> [-ot n] [-rt n] [-wl n] [-lg log] [-pg prog] and
 * the options passed to every job).  Jobs run in table order on ctx (NULL:
 * a context on device 0), the next jobs' host preparation overlapping the
 * GPU; the log (default ./master.log) gets the option echo, the JOB table
 * and the Worker table in the reference's format.  Returns MD_OK when the
 * queue ran (n_ok of n_jobs jobs ended with RET=0, and FILE=1 under -ot), or
 * an error for a missing table, log or PARAM= line. */
int md_table_mode(int argc, const char **argv);   /* 1 when argv has -tb */
int md_table_run(int argc, const char **argv, md_ctx *ctx, int *n_ok, int *n_jobs);
/* The argument vector of table job `job` (0-based) at attempt `retry`, one
 * argument per line, then "#out <file>" (the -ot field, empty without -ot);
 * job < 0 only counts the jobs into *n_jobs. */
int md_table_expand(int argc, const char **argv, int job, int retry, char *buf, int buflen, int *n_jobs);

/* .out consumers.  md_decoy_pdb writes the ligand PDB placed by pose number
 * `decoy` (1-based) of out_file (the decoygen tool, src/decoygen.cpp:39-149);
 * md_ligand_centres writes the placed ligand centre of every pose as
 * "x, y, z" lines or pseudo-atom HETATM records (pdb_format = 1) to dest
 * (NULL: standard output; the calcrg tool, src/calcrg.cpp:31-110). */
int md_decoy_pdb(const char *out_file, const char *ligand_pdb, int decoy, const char *dest_pdb);
int md_ligand_centres(const char *out_file, int pdb_format, const char *dest);

/* Receptor::electro (src/receptor.cpp:258-346) split by atom group: grids
 * holds ngroups * ng1^3 floats; atom l adds its field to grid group[l]
 * (atoms with group[l] outside [0, ngroups) are left out).  Same search
 * radius, dielectric, core mask and electrostatic ratio as the job's
 * receptor grid, so the groups sum to md_job_receptor_grids' imaginary part
 * up to the order of the float additions. */
int md_job_receptor_elec_groups(const md_job *job, const int *group, int ngroups, float *grids);
int md_job_centers(const md_job *job, float *rec_center, float *lig_center);
int md_job_rotation_angles(const md_job *job, float *theta);         /* 3 * n_rot */
float md_job_lig_core(const md_job *job);
/* Poses of the last md_job_run (n_rot * t, rotation-major) and the merged top. */
int md_job_poses(const md_job *job, md_pose *out);
int md_job_top(const md_job *job, md_pose *out);                      /* n_out */

#ifdef __cplusplus
}
#endif

#endif
