// Exit with XOR-network compiles still queued and running (no GPU needed):
// queues 40 matrices (each asked for twice) through xornet_launch (which returns before any CUDA
// call while a matrix is not compiled) and returns from main at once.  The
// process must exit cleanly: the compile workers are drained before NVRTC's
// own teardown.
#include <cstdio>
#include "kernels.h"
#include "xornet.h"
using namespace rsgpu;
int main() {
    DeviceInfo dev;
    dev.sm_count = 148;
    for (int s = 0; s < 40; s++) {
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
    printf("queued\n");
    return 0;
}
