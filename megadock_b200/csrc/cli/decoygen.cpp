// decoygen: the decoy complex of one pose of a .out file (MEGADOCK's tool of
// the same name and arguments, src/decoygen.cpp:126-149).
#include <cstdio>
#include <cstdlib>

#include "../../../include/md_b200.h"

int main(int argc, char **argv) {
    if (argc != 5) {
        std::printf("++ decoygen tool ++\n");
        std::printf("\n%s [decoy_filename] [used_ligand.pdb] [.outfile] [decoy no.]", argv[0]);
        std::printf("\n  **Note: files must be in PDB format.\n");
        return 255;
    }
    const int rc = md_decoy_pdb(argv[3], argv[2], (int)std::atof(argv[4]), argv[1]);
    if (rc) std::fprintf(stderr, "decoygen: cannot write decoy %s from %s (status %d)\n", argv[4], argv[3], rc);
    return rc ? 1 : 0;
}
