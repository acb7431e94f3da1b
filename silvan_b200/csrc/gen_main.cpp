// silvan_gen: writes one of the synthetic workloads as a `u v` edge list.
//   silvan_gen ba    N M SEED OUT
//   silvan_gen er    N MEANDEG SEED OUT
//   silvan_gen rmat  SCALE EDGEFACTOR SEED DIRECTED(0|1) OUT   (a,b,c = .57,.19,.19)
//   silvan_gen grid  SIDE DELFRAC SHORTCUTFRAC SEED OUT
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "gen.h"

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: silvan_gen ba|er|rmat|grid ...\n");
        return 1;
    }
    silvan::EdgeList e;
    const char *out = nullptr;
    if (!std::strcmp(argv[1], "ba") && argc == 6) {
        e = silvan::gen_ba(std::strtoul(argv[2], 0, 10), std::strtoul(argv[3], 0, 10),
                           std::strtoull(argv[4], 0, 10));
        out = argv[5];
    } else if (!std::strcmp(argv[1], "er") && argc == 6) {
        e = silvan::gen_er(std::strtoul(argv[2], 0, 10), std::strtod(argv[3], 0),
                           std::strtoull(argv[4], 0, 10));
        out = argv[5];
    } else if (!std::strcmp(argv[1], "rmat") && argc == 7) {
        e = silvan::gen_rmat(std::strtoul(argv[2], 0, 10), std::strtoul(argv[3], 0, 10), 0.57,
                             0.19, 0.19, std::strtoull(argv[4], 0, 10), std::atoi(argv[5]) != 0);
        out = argv[6];
    } else if (!std::strcmp(argv[1], "grid") && argc == 7) {
        e = silvan::gen_grid(std::strtoul(argv[2], 0, 10), std::strtod(argv[3], 0),
                             std::strtod(argv[4], 0), std::strtoull(argv[5], 0, 10));
        out = argv[6];
    } else {
        std::fprintf(stderr, "bad arguments\n");
        return 1;
    }
    if (!silvan::write_edge_list(out, e)) {
        std::fprintf(stderr, "cannot write %s\n", out);
        return 1;
    }
    std::fprintf(stderr, "%zu edges written to %s\n", e.size(), out);
    return 0;
}
