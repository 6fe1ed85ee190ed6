/* main.c -- the drop-in solver executable: `csu <case dir>/`, the reference's main.c:18-45 flow
 * (read the case, solve, write solution/solution2/restart/convergence/friction files) on the B200 engine. */
#include <stdio.h>
#include "csu_gpu.h"

int main(int argc, char** argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: %s <case directory ending in />\n", argv[0]);
        return 2;
    }
    int st = csu_run_case(argv[1], 1);
    if (st != CSU_OK) {
        fprintf(stderr, "csu: %s: %s\n", csu_strerror(st), csu_last_error());
        return 1;
    }
    return 0;
}
