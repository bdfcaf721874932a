// PDB reading, per-atom parameters, bounding box, grid sizing, grid
// coordinates and the rotation matrix.
//
// PDB contract (src/pdb_entry.cpp:18-105): ATOM/HETATM records; hydrogen
// lines (columns 77-78 == " H") are skipped; x/y/z from columns 31-38, 39-46,
// 47-54 (atof, stored as float); the table key is columns 12-21 with runs of
// spaces collapsed and the ends trimmed, e.g. "CA ALA".
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "../../../include/md_b200.h"
#include "host.h"

namespace mdb {

static std::string squeeze_spaces(const std::string &s0) {
    std::string s;
    s.reserve(s0.size());
    for (char c : s0) {
        if (c == ' ' && !s.empty() && s.back() == ' ') continue;
        s.push_back(c);
    }
    if (!s.empty() && s[0] == ' ') s.erase(0, 1);
    if (!s.empty() && s.back() == ' ') s.pop_back();
    return s;
}

static float lookup(const std::map<std::string, float> &m, const std::string &k, float dflt) {
    auto it = m.find(k);
    return it == m.end() ? dflt : it->second;
}

int read_molecule(const std::string &path, const Tables &tab, float grid_width, Molecule &m, std::string &err,
                  std::string &log) {
    (void)grid_width;
    m = Molecule();
    m.file = path;
    std::ifstream in(path);
    if (!in) {
        err = "[ERROR] PDB file [" + path + "] not open!!";
        return MD_ERR_IO;
    }
    std::string line;
    bool warned = false;
    while (std::getline(in, line)) {
        const std::string rec = line.substr(0, 6);
        if (rec != "ATOM  " && rec != "HETATM") continue;
        if (line.size() < 76) {
            // the reference's substr(76, 2) throws on such a line
            err = "[ERROR] PDB record shorter than 76 columns in " + path;
            return MD_ERR_IO;
        }
        if (line.compare(76, 2, " H") == 0 && line.substr(76, 2) == " H") {
            if (!warned) log += "# This PDB file contains hydrogen atom. MEGADOCK skips hydrogen atom line.\n";
            warned = true;
            continue;
        }
        for (int c = 0; c < 3; ++c) {
            const std::string f = line.substr(30 + 8 * c, 8);
            m.xyz.push_back((float)std::atof(f.c_str()));
        }
        m.atom_type.push_back(squeeze_spaces(line.substr(11, 10)));
    }
    const int na = (int)m.atom_type.size();
    m.radius.resize(na);
    m.charge.resize(na);
    m.ace.resize(na);
    for (int i = 0; i < na; ++i) {
        // defaults: carbon radius 1.8, neutral, no contact energy (src/parameter.cpp:425-470)
        m.radius[i] = lookup(tab.radius, m.atom_type[i], 1.8f);
        m.charge[i] = lookup(tab.charge, m.atom_type[i], 0.0f);
        m.ace[i] = lookup(tab.ace, m.atom_type[i], 0.0f);
    }
    // Protein::axis_edge (src/protein.cpp:67-111)
    for (int d = 0; d < 3; ++d) {
        m.edge[d][0] = 1.0e9f;
        m.edge[d][1] = -1.0e9f;
    }
    for (int i = 0; i < na; ++i)
        for (int d = 0; d < 3; ++d) {
            const float c = m.xyz[3 * i + d];
            if (c < m.edge[d][0]) m.edge[d][0] = c;
            if (c > m.edge[d][1]) m.edge[d][1] = c;
        }
    for (int d = 0; d < 3; ++d) m.center[d] = (float)((double)(m.edge[d][0] + m.edge[d][1]) / 2.0);
    if (na == 0) {
        err = "[ERROR] no ATOM records in " + path;
        return MD_ERR_IO;
    }
    return MD_OK;
}

std::vector<float> centred_coordinates(const Molecule &m) {
    float c[3];
    for (int d = 0; d < 3; ++d) c[d] = (float)((double)(m.edge[d][0] + m.edge[d][1]) / 2.0);
    std::vector<float> out(m.xyz.size());
    for (int i = 0; i < m.na(); ++i)
        for (int d = 0; d < 3; ++d) out[3 * i + d] = m.xyz[3 * i + d] - c[d];
    return out;
}

// Largest bounding-box edge (Control::autogridr, src/control.cpp:287-326).
static float receptor_extent(const Molecule &r) {
    float best = 0.0f;
    for (int d = 0; d < 3; ++d) {
        const float s = r.edge[d][1] - r.edge[d][0];
        if (s > best) best = s;
    }
    return best;
}

// Largest interatomic distance (Control::autogridl, src/control.cpp:329-379).
static float ligand_extent(const Molecule &l) {
    float best = 0.0f;
    const int na = l.na();
    for (int i = 0; i < na - 1; ++i) {
        const float x1 = l.xyz[3 * i], y1 = l.xyz[3 * i + 1], z1 = l.xyz[3 * i + 2];
        for (int j = i + 1; j < na; ++j) {
            const float dx = l.xyz[3 * j] - x1, dy = l.xyz[3 * j + 1] - y1, dz = l.xyz[3 * j + 2] - z1;
            const float d2 = dx * dx + dy * dy + dz * dz;
            if (d2 > best) best = d2;
        }
    }
    return std::sqrt(best);
}

int size_grids(const Params &p, const Tables &tab, Molecule &rec, Molecule &lig, std::string &err,
               std::string &log) {
    std::ostringstream lg;
    const float srec = receptor_extent(rec);
    const float slig = ligand_extent(lig);
    // float + 2.0 (double) * float margin, stored back to float
    const float need_rec = (float)(srec + 2.0 * p.grid_space_rec);
    const float need_lig = (float)(slig + 2.0 * p.grid_space_lig);
    lg << "Receptor max size = " << srec << "\nRequired voxel size = " << need_rec << "\n";
    lg << "Ligand max size = " << slig << "\nRequired voxel size = " << need_lig << "\n";
    if (!p.num_fft_flag) {
        auto it = tab.fft_sets.find(p.fft_base_set);
        if (it == tab.fft_sets.end()) {
            err = "unknown FFT size table -l " + std::to_string(p.fft_base_set);
            return MD_ERR_ARG;
        }
        auto pick = [&](float need) {
            int ng = 1 + int(need / p.grid_width);
            for (int v : it->second)
                if (v >= ng) return v;
            return ng;
        };
        rec.num_grid = pick(need_rec);
        lig.num_grid = pick(need_lig);
    } else {
        const float search_length = p.grid_width * p.num_grid;
        if (need_rec > search_length) {
            err = "[ERROR] Receptor data is too big!!";
            return MD_ERR_SIZE;
        }
        if (need_lig > search_length) {
            err = "[ERROR] Ligand data is too big!!";
            return MD_ERR_SIZE;
        }
        rec.num_grid = lig.num_grid = p.num_grid;
    }
    lg << "Number of grid = " << std::max(rec.num_grid, lig.num_grid) << "\n";
    log += lg.str();
    return MD_OK;
}

std::vector<float> grid_coordinates(int ng1, float grid_width) {
    std::vector<float> gc(ng1);
    const float search_length = grid_width * ng1;
    for (int i = 0; i < ng1; ++i) gc[i] = (float)(search_length * (-0.5 + (0.5 + i) / ng1));
    return gc;
}

void rotation_matrix(const float *th, float *m) {
    // float cos/sin of the float angles; products left to right
    const float c0 = std::cos(th[0]), s0 = std::sin(th[0]);
    const float c1 = std::cos(th[1]), s1 = std::sin(th[1]);
    const float c2 = std::cos(th[2]), s2 = std::sin(th[2]);
    m[0] = c0 * c2 - s0 * c1 * s2;    // r11
    m[1] = -c0 * s2 - s0 * c1 * c2;   // r12
    m[2] = s0 * s1;                   // r13
    m[3] = s0 * c2 + c0 * c1 * s2;    // r21
    m[4] = -s0 * s2 + c0 * c1 * c2;   // r22
    m[5] = -c0 * s1;                  // r23
    m[6] = s1 * s2;                   // r31
    m[7] = s1 * c2;                   // r32
    m[8] = c1;                        // r33
}

int write_out_file(const std::string &path, int nf1, float grid_width, const Molecule &rec, const Molecule &lig,
                   const Params &p, const std::vector<PoseRec> &top, std::string &err) {
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) {
        err = "[ERROR] Output file [" + path + "] not open!!";
        return MD_ERR_IO;
    }
    const float pi = (float)(4.0 * std::atan(1.0));
    std::fprintf(f, "%d\t%.2f\n", nf1, grid_width);
    std::fprintf(f, "\t%f\t%f\t%f\n", 0.0f, 0.0f, 0.0f);
    std::fprintf(f, "%s\t%f\t%f\t%f\n", p.rec_file.c_str(), rec.center[0], rec.center[1], rec.center[2]);
    std::fprintf(f, "%s\t%f\t%f\t%f\n", p.lig_file.c_str(), lig.center[0], lig.center[1], lig.center[2]);
    for (const PoseRec &r : top) {
        float th[3];
        for (int k = 0; k < 3; ++k) {
            th[k] = p.angles[3 * (size_t)r.rot + k];
            if (th[k] >= pi) th[k] = (float)(th[k] - pi * 2.0);
        }
        std::fprintf(f, "%f\t%f\t%f\t%d\t%d\t%d\t%.2f\n", th[0], th[1], th[2], r.i, r.j, r.k, r.score);
    }
    if (std::fclose(f) != 0) {
        err = "[ERROR] writing " + path;
        return MD_ERR_IO;
    }
    return MD_OK;
}

}  // namespace mdb
