// Consumers of the .out file: the decoy complex of one pose (MEGADOCK's
// decoygen tool, src/decoygen.cpp:39-149) and the ligand centre of every pose
// (its calcrg tool, src/calcrg.cpp:31-110).
//
// A pose (angles a, translation t in FFT cells, t >= N/2 read as t - N) puts
// a ligand atom x at  R(a) R(r0) (x - l) - t * spacing + c,  with l and c the
// ligand and receptor centres of the .out header and r0 its second line's
// angles.  The rotation matrix is formed in float (the float overloads of
// cos and sin), the products and sums in float without contraction, as the
// reference tools do, so their coordinates print identically.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/md_b200.h"

namespace {

struct OutHeader {
    int n = 0;
    float spacing = 0, r0[3] = {0, 0, 0}, rc[3] = {0, 0, 0}, lc[3] = {0, 0, 0};
};

struct OutPose {
    float a[3], t[3], score;
};

// z-x-z Euler rotation of one point
void rotate(const float in[3], float out[3], float psi, float theta, float phi) {
    using std::cos;   // float overloads, as the tools get them from <math.h> in C++
    using std::sin;
    const float r11 = cos(psi) * cos(phi) - sin(psi) * cos(theta) * sin(phi);
    const float r21 = sin(psi) * cos(phi) + cos(psi) * cos(theta) * sin(phi);
    const float r31 = sin(theta) * sin(phi);
    const float r12 = -cos(psi) * sin(phi) - sin(psi) * cos(theta) * cos(phi);
    const float r22 = -sin(psi) * sin(phi) + cos(psi) * cos(theta) * cos(phi);
    const float r32 = sin(theta) * cos(phi);
    const float r13 = sin(psi) * sin(theta);
    const float r23 = -cos(psi) * sin(theta);
    const float r33 = cos(theta);
    out[0] = r11 * in[0] + r12 * in[1] + r13 * in[2];
    out[1] = r21 * in[0] + r22 * in[1] + r23 * in[2];
    out[2] = r31 * in[0] + r32 * in[1] + r33 * in[2];
}

bool read_header(FILE *f, OutHeader &h) {
    char name[4096];
    return std::fscanf(f, "%d %f", &h.n, &h.spacing) == 2 &&
           std::fscanf(f, "%f %f %f", &h.r0[0], &h.r0[1], &h.r0[2]) == 3 &&
           std::fscanf(f, "%4095s %f %f %f", name, &h.rc[0], &h.rc[1], &h.rc[2]) == 4 &&
           std::fscanf(f, "%4095s %f %f %f", name, &h.lc[0], &h.lc[1], &h.lc[2]) == 4;
}

bool read_pose(FILE *f, OutPose &p) {
    return std::fscanf(f, "%f %f %f %f %f %f %f", &p.a[0], &p.a[1], &p.a[2], &p.t[0], &p.t[1], &p.t[2],
                       &p.score) == 7;
}

// placed position of a centred point for one pose
void place(const OutHeader &h, const OutPose &p, const float x[3], float out[3]) {
    float t1[3], t2[3];
    rotate(x, t1, h.r0[0], h.r0[1], h.r0[2]);
    rotate(t1, t2, p.a[0], p.a[1], p.a[2]);
    int t[3];
    for (int k = 0; k < 3; ++k) {
        t[k] = (int)p.t[k];
        if (t[k] >= h.n / 2) t[k] -= h.n;
        out[k] = t2[k] - t[k] * h.spacing + h.rc[k];
    }
}

}  // namespace

extern "C" {

int md_decoy_pdb(const char *out_file, const char *ligand_pdb, int decoy, const char *dest_pdb) {
    if (!out_file || !ligand_pdb || !dest_pdb || decoy < 1) return MD_ERR_ARG;
    FILE *fo = std::fopen(out_file, "r");
    if (!fo) return MD_ERR_IO;
    OutHeader h;
    OutPose p{};
    bool ok = read_header(fo, h);
    for (int i = 0; ok && i < decoy; ++i) ok = read_pose(fo, p);
    std::fclose(fo);
    if (!ok) return MD_ERR_ARG;
    FILE *in = std::fopen(ligand_pdb, "r");
    if (!in) return MD_ERR_IO;
    FILE *out = std::fopen(dest_pdb, "w");
    if (!out) {
        std::fclose(in);
        return MD_ERR_IO;
    }
    // the tool's own reading steps: 30 characters, then for ATOM/HETATM records
    // three 8-character coordinates and up to 59 more characters (the rest of
    // the record with its newline); TER, ENDMDL and "END   " records are copied
    char head[31], c[3][9], rest[60];
    while (std::fgets(head, sizeof head, in)) {
        if (!std::strncmp(head, "ATOM  ", 6) || !std::strncmp(head, "HETATM", 6)) {
            float x[3], y[3];
            for (int k = 0; k < 3; ++k) {
                if (!std::fgets(c[k], sizeof c[k], in)) c[k][0] = 0;
                x[k] = std::atof(c[k]) - h.lc[k];   // double difference, stored as float
            }
            if (!std::fgets(rest, sizeof rest, in)) rest[0] = 0;
            place(h, p, x, y);
            std::fprintf(out, "%s%8.3f%8.3f%8.3f%s", head, y[0], y[1], y[2], rest);
        } else if (!std::strncmp(head, "TER   ", 6) || !std::strncmp(head, "ENDMDL", 6) ||
                   !std::strncmp(head, "END   ", 6)) {
            if (!std::fgets(rest, sizeof rest, in)) rest[0] = 0;
            std::fprintf(out, "%s%s", head, rest);
        }
    }
    std::fclose(in);
    return std::fclose(out) == 0 ? MD_OK : MD_ERR_IO;
}

int md_ligand_centres(const char *out_file, int pdb_format, const char *dest) {
    if (!out_file) return MD_ERR_ARG;
    FILE *fo = std::fopen(out_file, "r");
    if (!fo) return MD_ERR_IO;
    OutHeader h;
    if (!read_header(fo, h)) {
        std::fclose(fo);
        return MD_ERR_ARG;
    }
    FILE *out = dest ? std::fopen(dest, "w") : stdout;
    if (!out) {
        std::fclose(fo);
        return MD_ERR_IO;
    }
    OutPose p;
    int i = 1;
    const float zero[3] = {0.f, 0.f, 0.f};
    while (read_pose(fo, p)) {
        float y[3];
        place(h, p, zero, y);
        if (pdb_format)
            std::fprintf(out, "HETATM %4d  S   RGS P%4d    %8.3f%8.3f%8.3f  1.00  1.00           S\n", i, i, y[0],
                         y[1], y[2]);
        else
            std::fprintf(out, "%7.3f, %7.3f, %7.3f\n", y[0], y[1], y[2]);
        if (++i == 10000) i = 0;
    }
    std::fclose(fo);
    if (dest) return std::fclose(out) == 0 ? MD_OK : MD_ERR_IO;
    std::fflush(out);
    return MD_OK;
}

}  // extern "C"
