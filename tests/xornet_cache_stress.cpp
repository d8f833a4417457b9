// Stress of the XOR-network compile cache on the CPU (no GPU needed): async queueing (through
// xornet_launch, which returns before any CUDA call while a matrix is not
// compiled) racing synchronous compiles (xornet_prepare) of the same and of
// new matrices, with background workers busy.  Must finish (no deadlock).
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>
#include "kernels.h"
#include "xornet.h"
using namespace rsgpu;
static GfMatArgs mk(int seed, int ni, int no) {
    GfMatArgs a{};
    a.n_in = ni; a.n_out = no; a.nbytes = 1 << 20;
    for (int i = 0; i < ni; i++) a.in[i] = reinterpret_cast<const uint8_t *>(uintptr_t(0x100000) * (i + 1));
    for (int o = 0; o < no; o++) a.out[o] = reinterpret_cast<uint8_t *>(uintptr_t(0x10000000) * (o + 1));
    for (int o = 0; o < no; o++) for (int i = 0; i < ni; i++) a.coef[o][i] = (uint8_t)((seed * 131 + o * 31 + i * 7) | 1);
    return a;
}
int main() {
    std::atomic<int> ok{0}, bad{0};
    DeviceInfo dev; dev.sm_count = 148;
    std::vector<std::thread> ts;
    for (int t = 0; t < 3; t++)
        ts.emplace_back([&, t] {   // async: queue 12 matrices each
            for (int s = 0; s < 12; s++) {
                GfMatArgs a = mk(100 * t + s, 6, 3);
                long long done = -1;
                xornet_launch(nullptr, dev, a, 0, false, &done);  // counted
                xornet_launch(nullptr, dev, a, 0, false, &done);  // queued
            }
        });
    for (int t = 0; t < 3; t++)
        ts.emplace_back([&, t] {   // sync: some overlap the queued ones, some new
            for (int s = 0; s < 10; s++) {
                GfMatArgs a = mk(s % 2 ? 100 * t + s : 7000 + 10 * t + s, 6, 3);
                (xornet_prepare(a, 0) ? ok : bad)++;
            }
        });
    for (auto &t : ts) t.join();
    int n = xornet_wait_idle();
    printf("sync ok=%d bad=%d compiled=%d\n", ok.load(), bad.load(), n);
    return bad.load() != 0;
}
