// Self-check of the fast correctly rounded division used by the FP64 kernels
// (mdiv / mrcp in multiphase-code_b200/csrc/hp_kernels.cuh) against the
// hardware IEEE division, on seeded random operands: dividends over
// 2^[-700, 700), divisors over 2^[-90, 90), with random mantissas plus
// all-ones, power-of-two and near-all-ones mantissas.  Prints
// "pairs N flagged F mismatches M" and exits 1 if M > 0.
// Built and run by tests/test_division.py.
#include <cstdint>
#include <cstdio>
#define HP_NS v_check
#define HP_R double
#define HP_LSQ_TABLE 1
#include "../multiphase-code_b200/csrc/hp_kernels.cuh"
using namespace hp::v_check;

__device__ unsigned long long g_mis, g_bad, g_n;
__device__ double g_example[8];

__device__ __forceinline__ unsigned long long xorshift(unsigned long long& s) {
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    return s;
}
__device__ double make_double(unsigned long long r, int e, int mode) {
    unsigned long long man = r & 0xfffffffffffffull;
    if (mode == 1) man = 0xfffffffffffffull;
    if (mode == 2) man = 0;
    if (mode == 3) man = 0xfffffffffffffull ^ (r & 0xffull);
    unsigned long long bits = ((r >> 63) << 63) | ((unsigned long long)(e + 1023) << 52) | man;
    return __longlong_as_double((long long)bits);
}
__global__ void k_check(unsigned long long seed, int iters) {
    unsigned long long s = seed ^ (0x9e3779b97f4a7c15ull * (blockIdx.x * blockDim.x + threadIdx.x + 1));
    unsigned long long nb = 0;
    for (int it = 0; it < iters; it++) {
        unsigned long long r1 = xorshift(s), r2 = xorshift(s), r3 = xorshift(s);
        int ea = (int)(r3 % 1400) - 700, eb = (int)((r3 >> 16) % 180) - 90;
        int ma = (r3 >> 32) % 8 == 0 ? (int)((r3 >> 40) % 4) : 0;
        int mb = (r3 >> 44) % 8 == 0 ? (int)((r3 >> 50) % 4) : 0;
        double a = make_double(r1, ea, ma), b = make_double(r2, eb, mb);
        if ((r3 >> 56) % 64 == 0) a = 0.0;
        unsigned bad = 0;
        double rb = mrcp<1>(b, bad);
        double q = mdiv<1>(a, b, rb, bad);
        if (bad) { nb++; continue; }
        if (__double_as_longlong(q) != __double_as_longlong(a / b)) {
            unsigned long long k = atomicAdd(&g_mis, 1ull);
            if (k < 4) { g_example[2 * k] = a; g_example[2 * k + 1] = b; }
        }
    }
    atomicAdd(&g_bad, nb);
    atomicAdd(&g_n, (unsigned long long)iters);
}
int main(int argc, char** argv) {
    int reps = argc > 1 ? atoi(argv[1]) : 2;
    for (int r = 0; r < reps; r++) {
        k_check<<<148 * 8, 256>>>(1234567ull + r, 4096);
        if (cudaDeviceSynchronize() != cudaSuccess) { printf("cuda error\n"); return 2; }
    }
    unsigned long long mis = 0, bad = 0, n = 0;
    double ex[8];
    cudaMemcpyFromSymbol(&mis, g_mis, 8);
    cudaMemcpyFromSymbol(&bad, g_bad, 8);
    cudaMemcpyFromSymbol(&n, g_n, 8);
    cudaMemcpyFromSymbol(ex, g_example, sizeof ex);
    printf("pairs %llu flagged %llu mismatches %llu\n", n, bad, mis);
    for (int i = 0; i < 4 && i < (int)mis; i++) printf("  a=%a b=%a\n", ex[2 * i], ex[2 * i + 1]);
    return mis != 0;
}
