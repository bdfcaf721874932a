// megadock-b200: the MEGADOCK command line (src/main.cpp, src/control.cpp)
// over the B200 pipeline.  Same flags (-R -L -o -N -t -F -v -D -r -e -d -a -b
// -f ...), same .out file; one GPU (device 0), no CPU fallback.  With -tb it
// is the table-mode driver (megadock-dp, src/mpidp.cpp) as one process.
#include <chrono>
#include <cstdio>

#include "../../../include/md_b200.h"

int main(int argc, char **argv) {
    if (md_table_mode(argc, (const char **)argv)) {
        // -tb: the table's jobs as a one-process queue (MEGADOCK's megadock-dp)
        int ok = 0, n = 0;
        const int rc = md_table_run(argc, (const char **)argv, nullptr, &ok, &n);
        if (rc) return rc == MD_ERR_USAGE ? 255 : 1;
        std::printf(" megadock-b200 table mode: %d of %d jobs ended normally\n", ok, n);
        return ok == n ? 0 : 1;
    }
    std::printf(" megadock-b200 (MEGADOCK 4.1.3 command line, B200 pipeline)\n\n");
    const auto t0 = std::chrono::steady_clock::now();
    md_job *job = nullptr;
    int rc = md_job_create(argc, (const char **)argv, &job);
    std::fputs(md_job_log(job), stdout);
    if (rc) {
        std::fprintf(stderr, "%s\n", md_job_error(job));
        md_job_destroy(job);
        return rc == MD_ERR_USAGE ? 255 : 1;
    }
    int ng1, nf1, nar, nal, nrot, t, nout;
    md_job_dims(job, &ng1, &nf1, &nar, &nal, &nrot, &t, &nout);
    std::printf("# receptor atoms %d, ligand atoms %d, FFT N = %d, rotations %d, t = %d\n", nar, nal, nf1, nrot, t);
    const auto t1 = std::chrono::steady_clock::now();
    rc = md_job_run(job, nullptr);
    const auto t2 = std::chrono::steady_clock::now();
    if (rc) {
        std::fprintf(stderr, "%s\n", md_job_error(job));
        md_job_destroy(job);
        return 1;
    }
    const double init = std::chrono::duration<double>(t1 - t0).count();
    const double dock = std::chrono::duration<double>(t2 - t1).count();
    std::printf("\nCPU time (initialize)         = %8.2f sec.\n", init);
    std::printf("Docking (receptor FFT + %d rotations) = %8.2f sec. (%.1f rotations/s)\n", nrot, dock, nrot / dock);
    std::printf("Output file = %s\n", md_job_out_file(job));
    md_job_destroy(job);
    return 0;
}
