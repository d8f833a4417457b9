// Compile policy of the XOR-network cache (no GPU needed), run with
// RSGPU_XORNET_CACHE_CAP=3: a matrix asked for once is not compiled, the
// second request queues it; synchronous compiles past the capacity evict the
// least recently used entries, so every one succeeds and the cache never
// holds more than three.
#include <cstdio>
#include "kernels.h"
#include "xornet.h"
using namespace rsgpu;
static GfMatArgs mk(int seed) {
    GfMatArgs a{};
    a.n_in = 5; a.n_out = 2; a.nbytes = 1 << 20;
    for (int i = 0; i < 5; i++) a.in[i] = reinterpret_cast<const uint8_t *>(uintptr_t(0x100000) * (i + 1));
    for (int o = 0; o < 2; o++) a.out[o] = reinterpret_cast<uint8_t *>(uintptr_t(0x10000000) * (o + 1));
    for (int o = 0; o < 2; o++) for (int i = 0; i < 5; i++) a.coef[o][i] = (uint8_t)((seed * 71 + o * 29 + i * 11) | 1);
    return a;
}
int main() {
    DeviceInfo dev; dev.sm_count = 148;
    long long done = -1;
    GfMatArgs a = mk(1);
    xornet_launch(nullptr, dev, a, 0, false, &done);
    const int after_one = xornet_wait_idle();
    xornet_launch(nullptr, dev, a, 0, false, &done);
    const int after_two = xornet_wait_idle();
    int ok = 0;
    for (int s = 2; s < 8; s++) ok += xornet_prepare(mk(s), 0) ? 1 : 0;
    const int held = xornet_wait_idle();
    printf("after_one=%d after_two=%d sync_ok=%d held=%d\n", after_one, after_two, ok, held);
    return (after_one == 0 && after_two == 1 && ok == 6 && held == 3) ? 0 : 1;
}
