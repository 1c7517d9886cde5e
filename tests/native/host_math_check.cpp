// Host-side check of two exact integer routines the kernels use (csrc/common.cuh):
//  * x87_mean(total, count) must equal (double)((long double)total / (long double)count),
//    the reference's histogram mean (src/wang_landau.cpp:349-361);
//  * fast_mod(x) must equal x % bound (Barrett reduction used by bounded(),
//    include/wl/rng.hpp:29-36);
//  * rng_step_back must invert Rng::next();
//  * the sweeps' bin floor: for a bin coordinate 0 <= q < 2^31, the sum q + 2^52 rounded toward
//    -infinity is 2^52 + floor(q), so its low word is floor(q) (bin_floor in walker_dev.cuh does
//    the add with __dadd_rd; here the host rounding mode stands in for it).
// Prints "ok <cases>" or the first mismatch.
#include <cfenv>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../replica_exchange_wang_landau_b200/csrc/common.cuh"

int main() {
    wlg::Rng rng;
    rng.seed(2024, 7);
    uint64_t cases = 0;
    for (int k = 0; k < 3000000; ++k) {
        const uint64_t a = 1 + rng.next() % (k % 3 == 0 ? 4096 : (k % 3 == 1 ? 64 : 1000000007ULL));
        uint64_t t = rng.next();
        switch (k % 5) {
            case 0: t %= 1000; break;
            case 1: t %= 1ULL << 40; break;
            case 2: t = (t % 100000) * a + (rng.next() % a); break;
            case 3: t >>= (rng.next() % 64); break;
            default: break;
        }
        const double want = static_cast<double>(static_cast<long double>(t) / static_cast<long double>(a));
        const double got = wlg::x87_mean(t, a);
        if (t != 0 && std::memcmp(&want, &got, 8) != 0) {
            std::printf("x87_mean mismatch total=%" PRIu64 " count=%" PRIu64 " want=%a got=%a\n", t, a, want, got);
            return 1;
        }
        ++cases;
    }
    const uint64_t bounds[] = {1, 2, 3, 7, 8, 27, 100, 512, 2458, 32768, 1000003, 2147483647ULL};
    for (uint64_t b : bounds) {
        const wlg::FastMod f = wlg::make_fastmod(b);
        for (int k = 0; k < 200000; ++k) {
            const uint64_t x = k < 10 ? ~0ULL - static_cast<uint64_t>(k) : rng.next();
            if (wlg::fast_mod(f, x) != x % b) {
                std::printf("fast_mod mismatch x=%" PRIu64 " bound=%" PRIu64 "\n", x, b);
                return 1;
            }
            ++cases;
        }
        if (f.threshold != (0ULL - b) % b) {
            std::printf("threshold mismatch bound=%" PRIu64 "\n", b);
            return 1;
        }
    }
    // rng_step_back inverts Rng::next() exactly
    for (int k = 0; k < 100000; ++k) {
        wlg::Rng a;
        a.seed(rng.next(), rng.next());
        const int steps = 1 + k % 9;
        wlg::Rng b = a;
        for (int s = 0; s < steps; ++s) (void)b.next();
        for (int s = 0; s < steps; ++s) wlg::rng_step_back(b);
        if (a.s0 != b.s0 || a.s1 != b.s1 || a.s2 != b.s2 || a.s3 != b.s3) {
            std::printf("rng_step_back mismatch at case %d\n", k);
            return 1;
        }
        ++cases;
    }
    // bin floor by a directed-rounding add
    {
        std::fesetround(FE_DOWNWARD);
        for (int k = 0; k < 2000000; ++k) {
            double q;
            const uint64_t r = rng.next();
            switch (k % 4) {
                case 0: q = static_cast<double>(r >> 33) * 0x1p-20; break;                  // fractional coordinates
                case 1: q = static_cast<double>(r % 100000); break;                          // exact integers
                case 2: q = std::nextafter(static_cast<double>(1 + r % 100000), 0.0); break;  // just below an integer
                default: q = static_cast<double>(r >> 33); break;                            // up to 2^31 - 1
            }
            volatile double a = q;
            volatile double sum = a + 0x1p52;
            const double s = sum;
            uint64_t bits;
            std::memcpy(&bits, &s, 8);
            const uint32_t low = static_cast<uint32_t>(bits & 0xffffffffULL);
            std::fesetround(FE_TONEAREST);
            const uint32_t want = static_cast<uint32_t>(std::floor(q));
            std::fesetround(FE_DOWNWARD);
            if (low != want) {
                std::fesetround(FE_TONEAREST);
                std::printf("bin floor mismatch q=%a low=%u want=%u\n", q, low, want);
                return 1;
            }
            ++cases;
        }
        std::fesetround(FE_TONEAREST);
    }
    std::printf("ok %" PRIu64 "\n", cases);
    return 0;
}
