// Background compiles queued before fork() must still finish: the child
// compiles a new matrix synchronously and waits for the queue it inherited;
// the parent waits for its own.  Host only: no GPU is touched.
#include <cstdio>
#include <sys/wait.h>
#include <unistd.h>
#include "kernels.h"
#include "xornet.h"
using namespace rsgpu;
static GfMatArgs mk(int seed) {
    GfMatArgs a{};
    a.n_in = 8; a.n_out = 3; a.nbytes = 1 << 20;
    for (int i = 0; i < 8; i++) a.in[i] = reinterpret_cast<const uint8_t *>(uintptr_t(0x100000) * (i + 1));
    for (int o = 0; o < 3; o++) a.out[o] = reinterpret_cast<uint8_t *>(uintptr_t(0x10000000) * (o + 1));
    for (int o = 0; o < 3; o++) for (int i = 0; i < 8; i++) a.coef[o][i] = (uint8_t)((seed * 53 + o * 31 + i * 7) | 1);
    return a;
}
int main() {
    DeviceInfo dev; dev.sm_count = 148;
    // each matrix asked for twice: the second request queues its compile
    for (int r = 0; r < 2; r++)
        for (int s = 0; s < 8; s++) { GfMatArgs a = mk(s); long long d; xornet_launch(nullptr, dev, a, 0, false, &d); }
    pid_t pid = fork();
    if (pid == 0) {
        GfMatArgs a = mk(1000);
        const bool ok = xornet_prepare(a, 0);
        const int n = xornet_wait_idle();
        printf("child ok=%d compiled=%d\n", ok, n);
        fflush(stdout);
        _exit(ok && n >= 9 ? 0 : 1);
    }
    int st = 0;
    waitpid(pid, &st, 0);
    const int n = xornet_wait_idle();
    printf("parent compiled=%d child_status=%d\n", n, WIFEXITED(st) ? WEXITSTATUS(st) : -1);
    return (WIFEXITED(st) && WEXITSTATUS(st) == 0 && n >= 8) ? 0 : 1;
}
