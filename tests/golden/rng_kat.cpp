// Generates known-answer vectors for the RNG layer from libstdc++ itself (GCC 13.3):
// std::mt19937_64 raw outputs, uniform_real_distribution<double>(0,1),
// normal_distribution<double>(0,1), uniform_int_distribution<int>(1,8),
// uniform_int_distribution<unsigned long>{0, b} and std::shuffle, for a few seeds.
// Build and run: g++ -O2 -o /tmp/rng_kat rng_kat.cpp && /tmp/rng_kat > rng_kat.txt
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <numeric>
#include <random>
#include <vector>
int main() {
    const std::uint64_t seeds[] = {104729ULL, 130363ULL, 433494437ULL, 88172645463325252ULL + 104729ULL, 1ULL};
    for (std::uint64_t s : seeds) {
        { std::mt19937_64 r(s); std::printf("raw %llu", (unsigned long long)s); for (int k = 0; k < 700; ++k) std::printf(" %llu", (unsigned long long)r()); std::printf("\n"); }
        { std::mt19937_64 r(s); std::uniform_real_distribution<double> U(0.0, 1.0); std::printf("u01 %llu", (unsigned long long)s); for (int k = 0; k < 400; ++k) std::printf(" %a", U(r)); std::printf("\n"); }
        { std::mt19937_64 r(s); std::normal_distribution<double> N(0.0, 1.0); std::printf("normal %llu", (unsigned long long)s); for (int k = 0; k < 400; ++k) std::printf(" %a", N(r)); std::printf("\n"); }
        { std::mt19937_64 r(s); std::uniform_int_distribution<int> B(1, 8); std::printf("ubin %llu", (unsigned long long)s); for (int k = 0; k < 400; ++k) std::printf(" %d", B(r)); std::printf("\n"); }
        { std::mt19937_64 r(s); std::printf("uint %llu", (unsigned long long)s); for (int k = 0; k < 400; ++k) { std::uniform_int_distribution<unsigned long> D{0, (unsigned long)(k % 37) + 1}; std::printf(" %lu", D(r)); } std::printf("\n"); }
        for (int n : {1, 2, 3, 8, 13, 30, 101}) {
            std::mt19937_64 r(s); std::vector<int> a(n); std::iota(a.begin(), a.end(), 0); std::shuffle(a.begin(), a.end(), r);
            std::printf("shuffle %llu %d", (unsigned long long)s, n); for (int x : a) std::printf(" %d", x); std::printf("\n");
        }
    }
}
