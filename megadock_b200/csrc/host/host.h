// Host-side model of a docking job: command line, force-field tables, PDB
// atoms, grid sizing, receptor grids and the .out writer.  Everything here is
// plain C++ compiled without FMA contraction, so every float result matches
// MEGADOCK's CPU code bit for bit.
#pragma once
#include <map>
#include <string>
#include <vector>

namespace mdb {

// Force-field tables keyed "<atom> <residue>" (src/parameter.cpp:425-470).
struct Tables {
    std::map<std::string, float> radius, charge, ace;
    std::map<int, std::vector<int>> fft_sets;   // -l table number -> ng1 sizes
};

// Directory holding the data assets (tables, rotation sets).
std::string data_dir();
bool load_tables(const std::string &dir, Tables &tab, std::string &err);
bool load_rotations(const std::string &dir, int nset, std::vector<float> &angles, std::string &err);

// Options of Parameter (src/parameter.h:34-118) that the docking path uses.
struct Params {
    std::string rec_file, lig_file, out_file, out_detail, out_csv, calc_id = "undefined";
    bool io_rec = false, io_lig = false, io_out = false;
    int detail_output = 0, calc_time_log = 0;
    int num_grid = 0, num_fft = 0, num_fft_flag = 0;
    int num_output = 2000, num_output_flag = 0;
    int thread_limit = 9999999, gpu_limit = 9999999;
    int score_func = 3, num_sort = 1;
    float elec_ratio = 1.0f, ace_ratio = 1.0f, grid_width = 1.2f;
    int rotation_set = 3600, fft_base_set = 11, lig_elec_serial = 0;
    int progress = 0, load_balance = 0, f1_flag = 0, f2_flag = 0;
    float rec_core = -45.0f, lig_core = 1.0f;
    float grid_space_rec = 8.0f, grid_space_lig = 3.0f;
    std::vector<float> angles;   // 3 per rotation
    int num_rot() const { return (int)(angles.size() / 3); }
};

// Parameter::initialize semantics; returns 0 or an MD_ERR_* code.
int parse_command_line(int argc, char **argv, Params &p, std::string &err, std::string &log);

// PDBEntry + Protein (src/pdb_entry.cpp:18-105, src/protein.cpp:19-131).
struct Molecule {
    std::string file;
    std::vector<std::string> atom_type;
    std::vector<float> xyz;   // 3 per atom
    std::vector<float> radius, charge, ace;
    float edge[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    float center[3] = {0, 0, 0};
    int num_grid = 0;
    int na() const { return (int)radius.size(); }
};

int read_molecule(const std::string &path, const Tables &tab, float grid_width, Molecule &m, std::string &err,
                  std::string &log);

// Grid sizing (src/control.cpp:287-464); returns 0 or an MD_ERR_* code.
int size_grids(const Params &p, const Tables &tab, Molecule &rec, Molecule &lig, std::string &err,
               std::string &log);

// Docking::rec_init grid coordinates (src/docking.cpp:139-142).
std::vector<float> grid_coordinates(int ng1, float grid_width);

// Centred coordinates: coordinate - (edge0 + edge1) / 2 (src/protein.cpp:114-131).
std::vector<float> centred_coordinates(const Molecule &m);

// Receptor rPSC+ACE and electrostatic grids (src/receptor.cpp:20-346).
void receptor_grids(const Molecule &rec, const Params &p, const std::vector<float> &gc, int ng1,
                    std::vector<float> &grid_r, std::vector<float> &grid_i);

// The electrostatic part alone (src/receptor.cpp:258-346) over the receptor
// core mask grid_r, into ngroups grids of ng1^3 (out): atom l contributes to
// grid group[l] (skipped when outside [0, ngroups)); group == nullptr puts
// every atom in grid 0, which is then the receptor's imaginary grid.
void receptor_electro(const Molecule &rec, const Params &p, const std::vector<float> &gc, int ng1,
                      const std::vector<float> &grid_r, const int *group, int ngroups, float *out);

// Rotation matrix of Docking::ligand_rotationz (src/docking.cpp:376-384).
void rotation_matrix(const float *theta, float *m9);

// .out writer (src/docking.cpp:399-453).
struct PoseRec {
    float score;
    int rot, i, j, k;
};
int write_out_file(const std::string &path, int nf1, float grid_width, const Molecule &rec, const Molecule &lig,
                   const Params &p, const std::vector<PoseRec> &top, std::string &err);

}  // namespace mdb
