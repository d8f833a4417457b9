// Exit with XOR-network compiles still queued and running (no GPU needed):
// queues matrices (each asked for twice) through xornet_launch (which
// returns before any CUDA call while a matrix is not compiled) and returns
// from main at once.  The process must exit cleanly: the compile workers are
// drained before NVRTC's own teardown.
//
//   exit_queued          40 matrices, exit during the process's first compiles
//   exit_queued warm     one matrix compiled and waited for first (NVRTC's
//                        own exit handlers exist by then), then 40, then exit
//
// Built with -shared -DRSGPU_EXIT_SHIM it exports queue_compiles(first, n)
// instead, for a Python host that loads it next to the package.
#include <cstdio>
#include <cstring>

#include "kernels.h"
#include "xornet.h"
using namespace rsgpu;

extern "C" int queue_compiles(int first, int n) {
    DeviceInfo dev;
    dev.sm_count = 148;
    for (int s = first; s < first + n; s++) {
        GfMatArgs a{};
        a.n_in = 10;
        a.n_out = 4;
        a.nbytes = 1 << 20;
        for (int i = 0; i < 10; i++) a.in[i] = reinterpret_cast<const uint8_t *>(uintptr_t(0x100000) * (i + 1));
        for (int o = 0; o < 4; o++) a.out[o] = reinterpret_cast<uint8_t *>(uintptr_t(0x10000000) * (o + 1));
        for (int o = 0; o < 4; o++)
            for (int i = 0; i < 10; i++) a.coef[o][i] = (uint8_t)((s * 131 + o * 31 + i * 7) | 1);
        long long done = -1;
        xornet_launch(nullptr, dev, a, 0, false, &done);  // counted
        xornet_launch(nullptr, dev, a, 0, false, &done);  // queued
    }
    return 0;
}

#ifndef RSGPU_EXIT_SHIM
int main(int argc, char **argv) {
    int first = 0;
    if (argc > 1 && strcmp(argv[1], "warm") == 0) {
        queue_compiles(1000, 1);
        xornet_wait_idle();
        first = 1;
    }
    queue_compiles(first, 40);
    printf("queued\n");
    return 0;
}
#endif
