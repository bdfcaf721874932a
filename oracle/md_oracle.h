/*
 * Test infrastructure (oracle side only; never linked into the product).
 * CPU restatement of MEGADOCK's per-rotation docking path, used as the checker
 * for the device pipeline.  See md_oracle.c for the reference citations.
 */
#ifndef MD_ORACLE_H
#define MD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Rotation matrix of Docking::ligand_rotationz for ZXZ angles theta[3]. */
void oracle_rotation_matrix(const float *theta, float *m9);

/* Rotated coordinates: out[3*l+d] = (m[3d]*x + m[3d+1]*y) + m[3d+2]*z. */
void oracle_rotate(int na, const float *xyz_centred, const float *m9, float *out);

/* Ligand rPSC (real) and charge (imaginary) grids for rotated coordinates. */
void oracle_ligand_grids(int na, const float *xyz_rot, const float *radius, const float *charge, int ng1,
                         float grid_width, const float *grid_coord, float delta, float *grid_r, float *grid_i);

/* Per-rotation top-t of a raw (unnormalised) real score grid of edge nf1:
 * scores[t], index3[3*t] (i, j, k). */
void oracle_score_sort(const float *raw, int nf1, int t, float *scores, int *index3);

#ifdef __cplusplus
}
#endif

#endif
