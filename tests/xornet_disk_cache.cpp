// Prepares (compiles now, or reads from RSGPU_KERNEL_CACHE) the XOR-network
// kernels of three coefficient tiles and prints how many NVRTC compilations
// ran and how many tiles have a kernel.  Host only: no GPU is touched.
#include <cstdio>
#include "kernels.h"
#include "xornet.h"
using namespace rsgpu;
int main() {
    int ok = 0;
    const int shapes[3][2] = {{10, 4}, {6, 3}, {17, 3}};
    for (int t = 0; t < 3; t++) {
        GfMatArgs a{};
        a.n_in = shapes[t][0];
        a.n_out = shapes[t][1];
        a.nbytes = 1 << 20;
        for (int o = 0; o < a.n_out; o++)
            for (int i = 0; i < a.n_in; i++) a.coef[o][i] = (uint8_t)((t * 97 + o * 29 + i * 13) | 1);
        ok += xornet_prepare(a, kModeWrite) ? 1 : 0;
    }
    printf("compiles=%d ok=%d\n", xornet_compile_count(), ok);
    return ok == 3 ? 0 : 1;
}
