// calcrg: the placed ligand centre of every pose of a .out file (MEGADOCK's
// tool of the same name and arguments, src/calcrg.cpp:82-110).
#include <cstdio>
#include <cstdlib>

#include "../../../include/md_b200.h"

int main(int argc, char **argv) {
    if (argc != 3) {
        std::printf("++ center points of ligand ++\n");
        std::printf("\n%s [.outfile] [isPDB? 0: csv,  1: pseudo PDB]\n", argv[0]);
        return 255;
    }
    const int rc = md_ligand_centres(argv[1], std::atoi(argv[2]), nullptr);
    if (rc) std::fprintf(stderr, "calcrg: cannot read %s (status %d)\n", argv[1], rc);
    return rc ? 1 : 0;
}
