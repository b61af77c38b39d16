// rng.h -- MT19937 (Matsumoto & Nishimura 1998; init_by_array 2002 revision),
// restated from the published algorithm. dgQuEST draws measurement outcomes
// from the classic mt19937ar generator (src/mt19937ar.c:61-154) through
// genrand_real1 (src/QuEST_common.c:106), so bit-exact outcomes need this
// exact generator, seeding and [0,1] scaling.
#pragma once

#include <cstdint>

namespace dgq {

class Mt19937 {
public:
    Mt19937() { seed(5489u); }

    void seed(uint32_t s) {
        mt_[0] = s;
        for (int i = 1; i < N; i++) mt_[i] = 1812433253u * (mt_[i - 1] ^ (mt_[i - 1] >> 30)) + (uint32_t) i;
        idx_ = N;
    }

    void seedArray(const unsigned long *key, int len) {
        seed(19650218u);
        int i = 1, j = 0;
        for (int k = (N > len ? N : len); k > 0; k--) {
            mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1664525u)) + (uint32_t) key[j] + (uint32_t) j;
            if (++i >= N) {
                mt_[0] = mt_[N - 1];
                i = 1;
            }
            if (++j >= len) j = 0;
        }
        for (int k = N - 1; k > 0; k--) {
            mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1566083941u)) - (uint32_t) i;
            if (++i >= N) {
                mt_[0] = mt_[N - 1];
                i = 1;
            }
        }
        mt_[0] = 0x80000000u;
    }

    uint32_t next() {
        if (idx_ >= N) twist();
        uint32_t y = mt_[idx_++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        return y;
    }

    // uniform on [0, 1], the 32-bit draw over 2^32 - 1
    double real1() { return (double) next() * (1.0 / 4294967295.0); }
    // uniform on [0, 1) with 53 bits: (a >> 5) * 2^26 + (b >> 6), over 2^53
    double res53() {
        const uint32_t a = next() >> 5, b = next() >> 6;
        return ((double) a * 67108864.0 + (double) b) * (1.0 / 9007199254740992.0);
    }

private:
    static constexpr int N = 624, M = 397;
    void twist() {
        for (int k = 0; k < N; k++) {
            const uint32_t y = (mt_[k] & 0x80000000u) | (mt_[(k + 1) % N] & 0x7fffffffu);
            mt_[k] = mt_[(k + M) % N] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        idx_ = 0;
    }
    uint32_t mt_[N];
    int idx_ = N;
};

}  // namespace dgq
