// Host check of xdiv_r (csrc/d3q19.cuh): correctly rounded x / y from the
// reciprocal RN(1/y), against the IEEE binary64 division of the host (SSE2).
// Compiled by tests/test_div_host.py with g++ -ffp-contract=off.
#include <cstdint>
#include <cstring>

#include "d3q19.cuh"

namespace {

uint64_t bits(double v) {
    uint64_t b;
    std::memcpy(&b, &v, sizeof(b));
    return b;
}

double from_bits(uint64_t b) {
    double v;
    std::memcpy(&v, &b, sizeof(v));
    return v;
}

// splitmix64
uint64_t next(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" {

// n random x (random sign and significand; exponent uniform in [emin, emax]) divided by y.
// Returns the number of results that differ from x / y bit for bit; *first_bad receives the
// first such x.
long long div_check_random(double y, long long n, uint64_t seed, int emin, int emax, double* first_bad) {
    const psc::Divisor d = psc::make_divisor(y);
    long long bad = 0;
    uint64_t s = seed;
    const uint64_t span = (uint64_t)(emax - emin + 1);
    for (long long i = 0; i < n; ++i) {
        const uint64_t r = next(s);
        const uint64_t e = (uint64_t)(emin + 1023 + (int64_t)(next(s) % span));
        const double x = from_bits((r & 0x800fffffffffffffull) | (e << 52));
        const double a = psc::xdiv_d(x, d), b = x / y;
        if (bits(a) != bits(b)) {
            if (bad == 0 && first_bad) *first_bad = x;
            ++bad;
        }
    }
    return bad;
}

// The same for a list of x; out[i] = xdiv_d(x[i], y).
long long div_check_list(double y, const double* xs, long long n, double* out) {
    const psc::Divisor d = psc::make_divisor(y);
    long long bad = 0;
    for (long long i = 0; i < n; ++i) {
        out[i] = psc::xdiv_d(xs[i], d);
        const double b = xs[i] / y;
        const bool same = bits(out[i]) == bits(b) || (out[i] != out[i] && b != b);  // any NaN matches a NaN
        bad += same ? 0 : 1;
    }
    return bad;
}

}  // extern "C"
