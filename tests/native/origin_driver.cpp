// Prints thy::tile_origin (kernels/kernels.h) for each group of four
// arguments "nx periodic sponge_left sponge_right", one origin per line.
// Used by tests/test_tile_origin.py; no GPU needed.
#include "kernels/kernels.h"

#include <cstdio>
#include <cstdlib>

int main(int argc, char **argv)
{
    for (int i = 1; i + 3 < argc; i += 4)
        std::printf("%d\n", thy::tile_origin(std::atoi(argv[i]), std::atoi(argv[i + 1]) != 0, std::atoi(argv[i + 2]),
                                             std::atoi(argv[i + 3])));
    return 0;
}
