// Drives egg::PerDevice (theeggman.jl_b200/csrc/egg_perdevice.h) with device indices directly, as a
// process holding two GPUs would: each device's value is set up once, by a set-up run for that
// device, and one device's value is never handed out for another.  Prints "ok" on success.
#include <cstdio>
#include <thread>
#include <vector>

#include "egg_perdevice.h"

static int fails = 0;
#define CHECK(c)                                                         \
    do {                                                                 \
        if (!(c)) {                                                      \
            std::printf("FAIL line %d: %s\n", __LINE__, #c);             \
            ++fails;                                                     \
        }                                                                \
    } while (0)

int main()
{
    egg::PerDevice<const void *> addr;
    int calls[egg::kMaxDevices] = {};
    // Stand-in for cudaGetSymbolAddress: device d's copy of a table lives at a distinct address.
    static char table_on[2][16];
    auto init = [&](int d, const void **out) {
        ++calls[d];
        *out = table_on[d];
        return 0;
    };
    const void *a0 = nullptr, *a1 = nullptr, *again = nullptr;
    CHECK(addr.get(0, &a0, init) == 0);
    CHECK(addr.get(1, &a1, init) == 0);
    CHECK(a0 == table_on[0] && a1 == table_on[1]);
    CHECK(addr.get(0, &again, init) == 0 && again == table_on[0]);
    CHECK(addr.get(1, &again, init) == 0 && again == table_on[1]);
    CHECK(calls[0] == 1 && calls[1] == 1);
    // A device that was never set up gets its own set-up, not device 0's value.
    CHECK(!addr.has(5));
    CHECK(addr.get(5, &again, [&](int d, const void **out) {
        ++calls[d];
        *out = &calls[d];
        return 0;
    }) == 0);
    CHECK(again == &calls[5] && calls[5] == 1);
    // A failing set-up caches nothing and is retried on the next call.
    int tries = 0;
    auto flaky = [&](int, const void **out) {
        ++tries;
        if (tries == 1) return 7;
        *out = table_on[0];
        return 0;
    };
    CHECK(addr.get(3, &again, flaky) == 7);
    CHECK(!addr.has(3));
    CHECK(addr.get(3, &again, flaky) == 0 && again == table_on[0] && tries == 2);
    // Indices outside the table are refused.
    CHECK(addr.get(-1, &again, init) == egg::PerDevice<const void *>::kBadDevice);
    CHECK(addr.get(egg::kMaxDevices, &again, init) == egg::PerDevice<const void *>::kBadDevice);
    // Many threads asking for the same new device run its set-up once.
    egg::PerDevice<int> shared;
    int setups = 0;
    std::vector<std::thread> th;
    for (int t = 0; t < 16; ++t)
        th.emplace_back([&] {
            int v = 0;
            shared.get(2, &v, [&](int, int *out) {
                ++setups;
                *out = 42;
                return 0;
            });
            if (v != 42) ++fails;
        });
    for (auto &t : th) t.join();
    CHECK(setups == 1);
    if (fails == 0) std::printf("ok\n");
    return fails == 0 ? 0 : 1;
}
