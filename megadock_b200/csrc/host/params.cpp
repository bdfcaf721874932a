// Command line, data tables and rotation sets.
//
// The option letters, defaults and cross-checks are MEGADOCK's
// (src/parameter.cpp:21-236 getopt loop, :266-308 defaults, :311-373 default
// output name, :376-422 rotation set and output clamp); they are part of the
// drop-in contract.  Errors are returned, never exit()ed.
#include <dlfcn.h>
#include <getopt.h>

#include <mutex>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "../../../include/md_b200.h"
#include "host.h"

namespace mdb {

std::string data_dir() {
    if (const char *e = std::getenv("MD_B200_DATA")) return e;
    Dl_info info;
    if (dladdr((void *)&data_dir, &info) && info.dli_fname) {
        std::string so = info.dli_fname;
        const size_t slash = so.rfind('/');
        std::string dir = slash == std::string::npos ? "." : so.substr(0, slash);
        return dir + "/../data";
    }
    return "megadock_b200/data";
}

static bool load_tsv(const std::string &path, std::map<std::string, float> &out, std::string &err) {
    std::ifstream in(path);
    if (!in) {
        err = "cannot open table " + path;
        return false;
    }
    std::string line;
    while (std::getline(in, line)) {
        const size_t tab = line.find('\t');
        if (tab == std::string::npos) continue;
        // decimal text -> double -> float, as the C++ initialiser converts it
        const float v = (float)std::strtod(line.c_str() + tab + 1, nullptr);
        out.emplace(line.substr(0, tab), v);   // first occurrence wins (map::insert)
    }
    return true;
}

bool load_tables(const std::string &dir, Tables &tab, std::string &err) {
    if (!load_tsv(dir + "/charmm_radius.tsv", tab.radius, err)) return false;
    if (!load_tsv(dir + "/charmm_charge.tsv", tab.charge, err)) return false;
    if (!load_tsv(dir + "/ace.tsv", tab.ace, err)) return false;
    std::ifstream in(dir + "/fft_tables.tsv");
    if (!in) {
        err = "cannot open " + dir + "/fft_tables.tsv";
        return false;
    }
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        int set;
        if (!(ss >> set)) continue;
        std::vector<int> v;
        int x;
        while (ss >> x) v.push_back(x);
        tab.fft_sets[set] = v;
    }
    return true;
}

bool load_rotations(const std::string &dir, int nset, std::vector<float> &angles, std::string &err) {
    const std::string path = dir + "/rotations_" + std::to_string(nset) + ".f32";
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) {
        err = "cannot open rotation set " + path;
        return false;
    }
    angles.assign((size_t)nset * 3, 0.f);
    const size_t got = std::fread(angles.data(), sizeof(float), angles.size(), f);
    std::fclose(f);
    if (got != angles.size()) {
        err = "short rotation set " + path;
        return false;
    }
    return true;
}

static std::string base_without_ext(std::string s) {
    const size_t slash = s.rfind('/');
    if (slash != std::string::npos) s = s.substr(slash + 1);
    const size_t dot = s.rfind('.');
    // std::string::substr(0, npos) keeps everything when there is no dot
    return s.substr(0, dot);
}

int parse_command_line(int argc, char **argv, Params &p, std::string &err, std::string &log) {
    // getopt keeps its state in globals: one parse at a time (the table mode
    // prepares jobs on several host threads)
    static std::mutex getopt_lock;
    std::lock_guard<std::mutex> hold(getopt_lock);
    p = Params();
    const std::string rb = "_r_b.pdb", lb = "_l_b.pdb", ru = "_r_u.pdb", lu = "_l_u.pdb";
    optind = 1;
    opterr = 0;
    int ch;
    std::ostringstream lg;
    while ((ch = getopt(argc, argv, "R:L:B:U:o:ON:t:E:a:b:e:d:F:v:Dhy:z:r:f:i:jkl:S:G:T:")) != -1) {
        switch (ch) {
        case 'R': p.rec_file = optarg; p.io_rec = true; break;
        case 'L': p.lig_file = optarg; p.io_lig = true; break;
        case 'B':
            p.rec_file = std::string(optarg) + rb;
            p.lig_file = std::string(optarg) + lb;
            p.io_rec = p.io_lig = true;
            break;
        case 'U':
            p.rec_file = std::string(optarg) + ru;
            p.lig_file = std::string(optarg) + lu;
            p.io_rec = p.io_lig = true;
            break;
        case 'o': {
            p.out_file = optarg;
            p.out_detail = p.out_file + ".detail";
            p.out_csv = p.out_file + ".csv";
            if (p.out_file.size() > 4 && p.out_file.substr(p.out_file.size() - 4) == ".out") {
                const std::string stem = p.out_file.substr(0, p.out_file.size() - 4);
                p.out_detail = stem + ".detail";
                p.out_csv = stem + ".csv";
            }
            p.io_out = true;
            break;
        }
        case 'O': p.detail_output = 1; break;
        case 'N':
            p.num_output = std::atoi(optarg);
            p.num_output_flag = 1;
            lg << "# Number of output = " << p.num_output << "\n";
            break;
        case 't':
            p.num_sort = std::atoi(optarg);
            lg << "# Set number of scores per one angle = " << p.num_sort << "\n";
            break;
        case 'E': p.calc_time_log = std::atoi(optarg); break;
        case 'i': p.calc_id = optarg; break;
        case 'e':
            p.elec_ratio = (float)std::atof(optarg);
            if (p.f1_flag == 1) {
                err = "Do not use -f 1 and -e option at the same time.";
                return MD_ERR_USAGE;
            }
            p.f1_flag = -1;
            lg << "# Set electric term ratio = " << p.elec_ratio << "\n";
            break;
        case 'd':
            p.ace_ratio = (float)std::atof(optarg);
            if (p.f1_flag == 1 || p.f2_flag == 1) {
                err = "Do not use -f 1 or 2 and -d option at the same time.";
                return MD_ERR_USAGE;
            }
            p.f1_flag = -1;
            p.f2_flag = -1;
            lg << "# Set ACE term ratio = " << p.ace_ratio << "\n";
            break;
        case 'a': p.rec_core = (float)std::atof(optarg); break;
        case 'b': p.lig_core = (float)std::atof(optarg); break;
        case 'F':
            p.num_fft = std::atoi(optarg);
            p.num_grid = p.num_fft / 2;
            p.num_fft_flag = 1;
            lg << "# Number of FFT N  = " << p.num_fft << "\n";
            break;
        case 'v':
            p.grid_width = (float)std::atof(optarg);
            lg << "# Set voxel size   = " << p.grid_width << "\n";
            break;
        case 'T':
            p.thread_limit = std::atoi(optarg);
            if (p.thread_limit < 1) {
                err = "Please set a positive number (Number of cores).";
                return MD_ERR_USAGE;
            }
            break;
        case 'G':
            p.gpu_limit = std::atoi(optarg);
            if (p.gpu_limit < 0) {
                err = "Please set a non-negative number (Number of GPUs you want to use).";
                return MD_ERR_USAGE;
            }
            break;
        case 'f': {
            const int sf = std::atoi(optarg);
            if (sf < 1 || sf > 3) {
                err = "score function must be 1, 2 or 3";
                return MD_ERR_USAGE;
            }
            if (sf == 1) {
                p.elec_ratio = 0.0f;
                p.ace_ratio = 0.0f;
                if (p.f1_flag == -1) {
                    err = "Do not use -f 1 and -e/-d option at the same time.";
                    return MD_ERR_USAGE;
                }
                p.f1_flag = 1;
            } else if (sf == 2) {
                p.ace_ratio = 0.0f;
                if (p.f2_flag == -1) {
                    err = "Do not use -f 2 and -d option at the same time.";
                    return MD_ERR_USAGE;
                }
                p.f2_flag = 1;
            }
            p.score_func = 3;   // the reference always scores with function 3
            break;
        }
        case 'r': p.rotation_set = std::atoi(optarg); break;
        case 'D':
            p.rotation_set = 54000;
            lg << "# Set 54,000 rotational angles (6 degree)\n";
            break;
        case 'j': p.progress = 1; break;
        case 'k': p.load_balance = 1; break;
        case 'S': p.lig_elec_serial = std::atoi(optarg); break;
        case 'l': p.fft_base_set = std::atoi(optarg); break;
        case 'h':
        default:
            err = "usage: megadock-b200 -R receptor.pdb -L ligand.pdb [-o out] [-N n] [-t n] [-F n] [-v w] "
                  "[-D | -r n] [-e x] [-d x] [-a x] [-b x] [-f 1|2|3]";
            return MD_ERR_USAGE;
        }
    }
    // Parameter::pdb_step (src/parameter.cpp:311-373)
    if (!p.io_rec) {
        err = "[ERROR] Receptor PDB file is not assignment!!";
        return MD_ERR_USAGE;
    }
    if (!p.io_lig) {
        err = "[ERROR] Ligand PDB file is not assignment!!";
        return MD_ERR_USAGE;
    }
    if (!p.io_out) {
        const std::string stem = base_without_ext(p.rec_file) + "-" + base_without_ext(p.lig_file);
        p.out_file = stem + ".out";
        p.out_detail = stem + ".detail";
        p.out_csv = stem + ".csv";
    }
    lg << "# Output file = " << p.out_file << "\n";
    // Parameter::parameter_set (src/parameter.cpp:376-422)
    const int sets[] = {3600, 54000, 1, 3, 24, 360};
    bool known = false;
    for (int s : sets) known |= (s == p.rotation_set);
    if (!known) {
        err = "[ERROR] Not support Rotation_angle_mode = " + std::to_string(p.rotation_set);
        return MD_ERR_ARG;
    }
    if (!load_rotations(data_dir(), p.rotation_set, p.angles, err)) return MD_ERR_IO;
    if (p.num_rot() * p.num_sort < p.num_output) {
        lg << "#[WARNING] Number of output file was changed from " << p.num_output;
        p.num_output = p.num_rot() * p.num_sort;
        lg << " to " << p.num_output << "\n";
    }
    if (p.num_sort < 1) {
        err = "number of scores per rotation (-t) must be positive";
        return MD_ERR_ARG;
    }
    log += lg.str();
    return MD_OK;
}

}  // namespace mdb
