// Table mode (-tb): MEGADOCK's MPI job farm (src/mpidp.cpp) as a one-process
// job queue on one GPU.
//
// Semantics kept from the reference:
//   * options -tb <table>, -ot <n> (field n is the job's output file; after
//     the job it is checked for existence), -rt <n> (retries; attempt r > 0
//     appends ".r" to field n), -wl <n> (failures after which a worker stops,
//     default 3), -lg <log> (default ./master.log), -pg <program> (accepted
//     and logged); every other argument is passed to each job before PARAM's
//     tokens (src/mpidp.cpp:132-251, :691-712);
//   * table lines: spaces in the first 7 characters are removed; TITLE= and
//     PARAM= (also Title=/title=, Param=/param=) set the title and the job
//     command; every other line is a job whose tab-separated fields replace
//     $1, $2, ... in PARAM in that order (src/mpidp.cpp:212-243, :786-823,
//     :856-878; the field count comes from the first job line);
//   * the job table and worker table of the log (src/mpidp.cpp:880-914).
// Differences: one worker (the GPU, WID=1) runs the jobs in table order;
// host preparation of the next jobs (PDB reading, grid sizing, receptor
// grids) runs on host threads while the GPU docks the current one.  Attempts
// follow the reference's order for one worker: every job once, then the
// failed ones again (round r uses the ".r" suffix) up to -rt rounds; the
// worker stops after -wl failures.
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <future>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/md_b200.h"
#include "host.h"

namespace {

struct TableSpec {
    std::string table_file, log_file = "./master.log", program;
    std::string title = "MasterProc", param = "MPIDP";
    int out_option = 0, ntry = 0, worker_life = 3;
    std::vector<std::string> app_args;   // argv[0] and every non-table option
    std::vector<std::string> rows;       // job lines
    int nfields = 0;                     // fields per job line (from the first)
    std::string log;                     // option and table echo for the log
};

bool table_opt(const char *a) {
    return !std::strncmp(a, "-tb", 3) || !std::strncmp(a, "-ot", 3) || !std::strncmp(a, "-rt", 3) ||
           !std::strncmp(a, "-wl", 3) || !std::strncmp(a, "-pg", 3) || !std::strncmp(a, "-lg", 3);
}

// spaces at positions below ip are removed, first to last (Mpidp::erase_space)
std::string erase_space(std::string s, size_t ip) {
    while (true) {
        const size_t n = s.find(' ');
        if (n == std::string::npos || n >= ip) break;
        s.erase(n, 1);
    }
    return s;
}

std::vector<std::string> split(const std::string &s, char sep) {   // strtok: empty tokens skipped
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && s[i] == sep) ++i;
        size_t j = i;
        while (j < s.size() && s[j] != sep) ++j;
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j;
    }
    return out;
}

std::string replace_all(const std::string &s, const std::string &from, const std::string &to) {
    std::string out;
    size_t pos = 0, prev = 0;
    while ((pos = s.find(from, pos)) != std::string::npos) {
        out.append(s, prev, pos - prev);
        out += to;
        pos += from.size();
        prev = pos;
    }
    out.append(s, prev, std::string::npos);
    return out;
}

int parse_table(int argc, const char **argv, TableSpec &t, std::string &err) {
    std::ostringstream lg;
    for (int i = 1; i < argc; ++i) {
        if (!table_opt(argv[i])) continue;
        if (i + 1 >= argc) {
            err = std::string("option ") + argv[i] + " needs a value";
            return MD_ERR_USAGE;
        }
        const char *v = argv[i + 1];
        if (!std::strncmp(argv[i], "-tb", 3)) {
            t.table_file = v;
            lg << "Table file    : -tb " << v << "\n";
        } else if (!std::strncmp(argv[i], "-ot", 3)) {
            t.out_option = std::atoi(v);
            lg << "Output option : -ot " << t.out_option << "\n";
        } else if (!std::strncmp(argv[i], "-rt", 3)) {
            t.ntry = std::atoi(v);
            lg << "Retry option  : -rt " << t.ntry << "\n";
        } else if (!std::strncmp(argv[i], "-wl", 3)) {
            t.worker_life = std::atoi(v);
            lg << "Worker life   : -wl " << t.worker_life << "\n";
        } else if (!std::strncmp(argv[i], "-pg", 3)) {
            t.program = v;
            lg << "Program name  : -pg " << v << "\n";
        } else {
            t.log_file = v;
            lg << "Log file      : -lg " << v << "\n";
        }
        ++i;
    }
    t.app_args.push_back(argc > 0 ? argv[0] : "megadock-b200");
    bool other = false;
    for (int i = 1; i < argc; ++i) {
        if (table_opt(argv[i])) {
            ++i;
            continue;
        }
        if (!other) lg << "Other options :";
        other = true;
        lg << " " << argv[i];
        t.app_args.push_back(argv[i]);
    }
    if (other) lg << "\n";
    lg << "\n";
    if (t.table_file.empty()) {
        err = "no table file (-tb)";
        return MD_ERR_USAGE;
    }
    std::ifstream in(t.table_file);
    if (!in) {
        err = "[ERROR] Table file [" + t.table_file + "] was not opened!!";
        return MD_ERR_IO;
    }
    std::string line;
    while (std::getline(in, line)) {
        line = erase_space(line, 7);
        const std::string head = line.substr(0, 6);
        if (head == "TITLE=" || head == "Title=" || head == "title=") {
            t.title = line.substr(6);
            lg << "TITLE=" << t.title << "\n";
        } else if (head == "PARAM=" || head == "Param=" || head == "param=") {
            t.param = line.substr(6);
            lg << "PARAM=" << t.param << "\n";
        } else {
            t.rows.push_back(line);
        }
    }
    lg << "\n";
    if (!t.rows.empty()) t.nfields = (int)std::count(t.rows[0].begin(), t.rows[0].end(), '\t') + 1;
    if (t.param == "MPIDP") {
        err = "[ERROR] [PARAM=] was not found in table file!!";
        return MD_ERR_USAGE;
    }
    t.log = lg.str();
    return MD_OK;
}

// The job's argument vector for attempt `retry` (Mpidp::for_worker): PARAM with
// $1..$n replaced by the row's fields, field -ot suffixed ".retry" on retries.
int job_args(const TableSpec &t, int job, int retry, std::vector<std::string> &args, std::string &out_file,
             std::string &err) {
    const std::vector<std::string> f = split(t.rows[job], '\t');
    if ((int)f.size() < t.nfields) {
        err = "table line " + std::to_string(job + 1) + " has fewer fields than the first job line";
        return MD_ERR_ARG;
    }
    std::string p = t.param;
    out_file.clear();
    for (int i = 0; i < t.nfields; ++i) {
        std::string v = f[i];
        if (t.out_option == i + 1) {
            if (retry) v += "." + std::to_string(retry);
            out_file = v;
        }
        p = replace_all(p, "$" + std::to_string(i + 1), v);
    }
    args = t.app_args;
    for (const std::string &tok : split(p, ' ')) args.push_back(tok);
    return MD_OK;
}

struct Prepared {
    md_job *job = nullptr;
    int rc = MD_OK;
    std::string out_file, err;
};

Prepared prepare(const TableSpec &t, int job, int retry) {
    Prepared p;
    std::vector<std::string> args;
    p.rc = job_args(t, job, retry, args, p.out_file, p.err);
    if (p.rc) return p;
    std::vector<const char *> av;
    for (const std::string &a : args) av.push_back(a.c_str());
    p.rc = md_job_create((int)av.size(), av.data(), &p.job);
    if (p.rc) p.err = md_job_error(p.job);
    return p;
}

struct Attempt {
    int end = 0, ret = -1, file = 0;
};

}  // namespace

extern "C" {

int md_table_mode(int argc, const char **argv) {
    for (int i = 1; i < argc; ++i)
        if (argv[i] && !std::strncmp(argv[i], "-tb", 3)) return 1;
    return 0;
}

int md_table_expand(int argc, const char **argv, int job, int retry, char *buf, int buflen, int *n_jobs) {
    TableSpec t;
    std::string err;
    int rc = parse_table(argc, argv, t, err);
    if (rc) return rc;
    if (n_jobs) *n_jobs = (int)t.rows.size();
    if (job < 0) return MD_OK;
    if (job >= (int)t.rows.size() || retry < 0 || !buf || buflen < 1) return MD_ERR_ARG;
    std::vector<std::string> args;
    std::string out_file;
    if ((rc = job_args(t, job, retry, args, out_file, err))) return rc;
    std::string s;
    for (const std::string &a : args) s += a + "\n";
    s += "#out " + out_file;
    if ((int)s.size() + 1 > buflen) return MD_ERR_ARG;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return MD_OK;
}

int md_table_run(int argc, const char **argv, md_ctx *ctx, int *n_ok, int *n_jobs) {
    TableSpec t;
    std::string err;
    int rc = parse_table(argc, argv, t, err);
    if (rc) {
        std::fprintf(stderr, "%s\n", err.c_str());
        return rc;
    }
    std::ofstream log(t.log_file);
    if (!log) {
        std::fprintf(stderr, "[ERROR] Log file [%s] was not opened!!\n", t.log_file.c_str());
        return MD_ERR_IO;
    }
    const auto t0 = std::chrono::steady_clock::now();
    log << " megadock-b200 table mode (one process, one GPU worker)\n\n#RANK = 2\n#Node = 1 (#RANK/Node = 2)\n\n";
    log << t.log;
    log.flush();
    md_ctx *own = nullptr;
    if (!ctx) {
        if ((rc = md_ctx_create(0, &own))) {
            std::fprintf(stderr, "cannot create a device context on device 0\n");
            return rc;
        }
        ctx = own;
    }
    const int nj = (int)t.rows.size();
    std::vector<std::vector<Attempt>> att(nj);
    std::vector<int> exec(nj, 0);
    std::vector<bool> done(nj, false);
    std::vector<std::string> worker_names;   // jobs in the order the worker ran them
    std::vector<int> worker_codes;
    int failures = 0;
    bool stopped = false;
    // host preparation ahead of the GPU: up to `ahead` jobs of round 0 in flight
    const int ahead = std::max(1, std::min(8, (int)std::thread::hardware_concurrency()));
    std::deque<std::future<Prepared>> pending;
    int next = 0;
    auto top_up = [&]() {
        while (next < nj && (int)pending.size() < ahead) {
            const int j = next++;
            pending.push_back(std::async(std::launch::async, [&t, j]() { return prepare(t, j, 0); }));
        }
    };
    auto name_of = [](int j) {
        char b[16];
        std::snprintf(b, sizeof b, "%05d\t", j + 1);
        return std::string(b);
    };
    for (int round = 0; round <= t.ntry && !stopped; ++round) {
        for (int j = 0; j < nj && !stopped; ++j) {
            if (done[j] || exec[j] != round) continue;
            Prepared p;
            if (round == 0) {
                top_up();
                p = pending.front().get();
                pending.pop_front();
                top_up();
            } else {
                p = prepare(t, j, round);
            }
            ++exec[j];
            Attempt a;
            a.end = 1;
            a.ret = p.rc;
            if (!p.rc) {
                a.ret = md_job_run(p.job, ctx);
                if (a.ret) std::fprintf(stderr, "job %d: %s\n", j + 1, md_job_error(p.job));
            } else {
                std::fprintf(stderr, "job %d: %s\n", j + 1, p.err.c_str());
            }
            md_job_destroy(p.job);
            if (t.out_option) {
                struct stat st;
                a.file = stat(p.out_file.c_str(), &st) == 0 ? 1 : -1;
            }
            att[j].push_back(a);
            worker_names.push_back(name_of(j));
            worker_codes.push_back(1);
            const bool ok = a.ret == 0 && (a.file == 1 || t.out_option == 0);
            if (t.ntry == 0 || ok) {
                done[j] = true;
            } else if (++failures >= t.worker_life) {
                std::fprintf(stderr, "[Warning] Worker 1 starts sleeping.\n[ERROR] All wokers were stoped!!\n");
                stopped = true;
            }
        }
    }
    // jobs never reached keep their prepared state out of the way
    while (!pending.empty()) {
        Prepared p = pending.front().get();
        pending.pop_front();
        md_job_destroy(p.job);
    }
    int ok_jobs = 0;
    log << "JOB table :\n";
    for (int j = 0; j < nj; ++j) {
        log << name_of(j) << " EXEC=" << exec[j];
        for (const Attempt &a : att[j])
            log << " (WID=1 END=" << a.end << " RET=" << a.ret << " FILE=" << a.file << ")";
        log << "\n";
        if (!att[j].empty()) {
            const Attempt &a = att[j].back();
            if (a.ret == 0 && (a.file == 1 || t.out_option == 0)) ++ok_jobs;
        }
    }
    log << "\nWorker table :\nno.\t#exec\tdetail\n1\t" << worker_names.size();
    for (size_t k = 0; k < worker_names.size(); ++k) log << "\t" << worker_names[k] << "\t" << worker_codes[k];
    log << "\n";
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    log << "\nElapsed time  = " << secs << " sec.\n";
    if (own) md_ctx_destroy(own);
    if (n_ok) *n_ok = ok_jobs;
    if (n_jobs) *n_jobs = nj;
    return MD_OK;
}

}  // extern "C"
