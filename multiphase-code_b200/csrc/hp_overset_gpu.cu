// hp_overset_gpu.cu -- hp_overset_build with its searches on the device.
//
// Same tables as hp_overset_build (hp_overset.cpp), bit for bit: the host
// marks the fringe and sizes the grids (hp_ov::prepare, O(cells)), and the
// device does the rest:
//
//   binning   every field tet of a block is registered in the grid cells its
//             bounding box spans (count, exclusive scan, fill);
//   donor     one thread per fringe cell tests the tets of its grid cell and
//             keeps the lowest id that contains the centroid (the host walks
//             ascending lists and stops at the first; the minimum over the
//             cell is the same tet);
//   fallback  one block per fringe cell that no tet contains: the field cell
//             of the other block with the nearest centroid, ties to the
//             lowest id (the host's first strict minimum in ascending order);
//   weights   one thread per fringe cell: the candidate rings and the tet of
//             four candidate centroids chosen by the host's rules.
//
// The arithmetic is the host's (hp_ov::bary, the same centroid and distance
// expressions), compiled without contraction, so every comparison and weight
// comes out identical.  Allocates and frees its own device buffers; runs on
// the current device and a stream of its own.
#include <cuda_runtime.h>

#include <climits>
#include <cstdlib>
#include <cstring>
#include <cub/device/device_scan.cuh>
#include <vector>

#include "../../include/hydraphase.h"
#include "hp_overset_common.h"

namespace {

struct DMesh {
    const double *x, *y, *z;
    const int32_t* elem;   // [neles][9], 1-based ids
    int neles;
};

__device__ __forceinline__ const int32_t* row(const DMesh& M, int e) { return M.elem + 9 * (size_t)(e - 1); }
__device__ __forceinline__ void node(const DMesh& M, int n, double p[3]) {
    p[0] = M.x[n - 1]; p[1] = M.y[n - 1]; p[2] = M.z[n - 1];
}
__device__ __forceinline__ void centroid(const DMesh& M, int e, double c[3]) {
    const int32_t* r = row(M, e);
    c[0] = 0.25 * (M.x[r[0] - 1] + M.x[r[1] - 1] + M.x[r[2] - 1] + M.x[r[3] - 1]);
    c[1] = 0.25 * (M.y[r[0] - 1] + M.y[r[1] - 1] + M.y[r[2] - 1] + M.y[r[3] - 1]);
    c[2] = 0.25 * (M.z[r[0] - 1] + M.z[r[1] - 1] + M.z[r[2] - 1] + M.z[r[3] - 1]);
}

// Grid cell range [a, b] per axis of tet t's bounding box.
__device__ __forceinline__ void span(const DMesh& M, const hp_ov::GridParams& g, int t, int a[3], int b[3]) {
    double bl[3] = {1e300, 1e300, 1e300}, bh[3] = {-1e300, -1e300, -1e300};
    for (int q = 0; q < 4; q++) {
        double p[3];
        node(M, row(M, t)[q], p);
        for (int d = 0; d < 3; d++) { bl[d] = fmin(bl[d], p[d]); bh[d] = fmax(bh[d], p[d]); }
    }
    for (int d = 0; d < 3; d++) { a[d] = hp_ov::grid_index(g, d, bl[d]); b[d] = hp_ov::grid_index(g, d, bh[d]); }
}

__device__ __forceinline__ size_t gcell(const hp_ov::GridParams& g, int i, int j, int k) {
    return ((size_t)i * g.n[1] + j) * g.n[2] + k;
}

__global__ void k_bin_count(DMesh M, hp_ov::GridParams g, const int* field, int nfield, int* cnt) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfield) return;
    int a[3], b[3];
    span(M, g, field[f], a, b);
    for (int i = a[0]; i <= b[0]; i++)
        for (int j = a[1]; j <= b[1]; j++)
            for (int k = a[2]; k <= b[2]; k++) atomicAdd(cnt + gcell(g, i, j, k), 1);
}

__global__ void k_bin_fill(DMesh M, hp_ov::GridParams g, const int* field, int nfield, const int* start, int* fill,
                           int* items) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfield) return;
    const int t = field[f];
    int a[3], b[3];
    span(M, g, t, a, b);
    for (int i = a[0]; i <= b[0]; i++)
        for (int j = a[1]; j <= b[1]; j++)
            for (int k = a[2]; k <= b[2]; k++) {
                const size_t c = gcell(g, i, j, k);
                items[start[c] + atomicAdd(fill + c, 1)] = t;
            }
}

struct Bins {
    hp_ov::GridParams g;
    const int* start;   // [ncell + 1]
    const int* items;
    int nfield;
};

// Lowest-id field tet of the other block containing the fringe centroid; 0
// if none (or if that block has no field cell).
__global__ void k_donor(DMesh M, const int* block, const int* fr, int nf, Bins b0, Bins b1, int* donor) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int e = fr[f];
    const Bins& B = block[e - 1] == 0 ? b1 : b0;
    int D = INT_MAX;
    if (B.nfield > 0) {
        double xp[3];
        centroid(M, e, xp);
        const size_t c = gcell(B.g, hp_ov::grid_index(B.g, 0, xp[0]), hp_ov::grid_index(B.g, 1, xp[1]),
                               hp_ov::grid_index(B.g, 2, xp[2]));
        for (int it = B.start[c]; it < B.start[c + 1]; it++) {
            const int t = B.items[it];
            if (t >= D) continue;
            const int32_t* r = row(M, t);
            double p[4][3], lam[4];
            for (int q = 0; q < 4; q++) node(M, r[q], p[q]);
            if (hp_ov::bary(p[0], p[1], p[2], p[3], xp, lam) == 0.0) continue;
            if (lam[0] >= -1e-10 && lam[1] >= -1e-10 && lam[2] >= -1e-10 && lam[3] >= -1e-10) D = t;
        }
    }
    donor[f] = D == INT_MAX ? 0 : D;
}

// Nearest field centroid of the other block for the fringe cells listed in
// miss (one block each): ties go to the lowest id.
__global__ void __launch_bounds__(256) k_nearest(DMesh M, const int* block, const int* fr, const int* miss,
                                                 const int* field0, int n0, const int* field1, int n1, int* donor) {
    const int f = miss[blockIdx.x];
    const int e = fr[f];
    const int* field = block[e - 1] == 0 ? field1 : field0;
    const int n = block[e - 1] == 0 ? n1 : n0;
    double xp[3];
    centroid(M, e, xp);
    double best = 0.0;
    int bid = INT_MAX;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int t = field[k];
        double cc[3];
        centroid(M, t, cc);
        const double d2 = (cc[0] - xp[0]) * (cc[0] - xp[0]) + (cc[1] - xp[1]) * (cc[1] - xp[1]) +
                          (cc[2] - xp[2]) * (cc[2] - xp[2]);
        if (bid == INT_MAX || d2 < best || (d2 == best && t < bid)) { best = d2; bid = t; }
    }
    __shared__ double sb[256];
    __shared__ int si[256];
    sb[threadIdx.x] = best;
    si[threadIdx.x] = bid;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double ob = sb[threadIdx.x + s];
            const int oi = si[threadIdx.x + s];
            const int mi = si[threadIdx.x];
            if (oi != INT_MAX && (mi == INT_MAX || ob < sb[threadIdx.x] || (ob == sb[threadIdx.x] && oi < mi))) {
                sb[threadIdx.x] = ob;
                si[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) donor[f] = si[0] == INT_MAX ? 0 : si[0];
}

// Candidate rings and barycentric weights (the host's rules, hp_overset.cpp).
__global__ void k_weights(DMesh M, const int* block, const int* iblank, const int* fr, int nf, const int* donor,
                          int32_t* dn_out, double* w_out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int e = fr[f], B = 1 - block[e - 1], D = donor[f];
    int32_t* dn = dn_out + 4 * (size_t)f;
    double* w = w_out + 4 * (size_t)f;
    if (!D) {
        dn[0] = dn[1] = dn[2] = dn[3] = e;
        w[0] = 1.0; w[1] = w[2] = w[3] = 0.0;
        return;
    }
    dn[0] = dn[1] = dn[2] = dn[3] = D;
    w[0] = 1.0; w[1] = w[2] = w[3] = 0.0;
    double xp[3];
    centroid(M, e, xp);
    int cand[17], m = 0;
    cand[m++] = D;
    for (int ring = 0, lo = 0; ring < 2; ring++) {
        int hi = m;
        for (int a = lo; a < hi; a++)
            for (int k = 0; k < 4 && m < 17; k++) {
                int n = row(M, cand[a])[4 + k];
                if (n > M.neles || iblank[n - 1] != 1 || block[n - 1] != B) continue;
                bool seen = false;
                for (int q = 0; q < m; q++) seen |= (cand[q] == n);
                if (!seen) cand[m++] = n;
            }
        lo = hi;
    }
    double cc[17][3];
    for (int a = 0; a < m; a++) centroid(M, cand[a], cc[a]);
    double best_in = 0.0, best_out = -1.0e300;
    bool have_in = false;
    for (int i = 0; i < m; i++)
        for (int j = i + 1; j < m; j++)
            for (int k = j + 1; k < m; k++)
                for (int l = k + 1; l < m; l++) {
                    double lam[4];
                    if (hp_ov::bary(cc[i], cc[j], cc[k], cc[l], xp, lam) == 0.0) continue;
                    const double sc = hp_ov::mn2(hp_ov::mn2(hp_ov::mn2(lam[0], lam[1]), lam[2]), lam[3]);
                    const int id[4] = {i, j, k, l};
                    if (sc >= -1e-12) {
                        double s2 = 0.0;
                        for (int q = 0; q < 4; q++)
                            s2 = s2 + ((cc[id[q]][0] - xp[0]) * (cc[id[q]][0] - xp[0]) +
                                       (cc[id[q]][1] - xp[1]) * (cc[id[q]][1] - xp[1]) +
                                       (cc[id[q]][2] - xp[2]) * (cc[id[q]][2] - xp[2]));
                        if (!have_in || s2 < best_in) {
                            have_in = true; best_in = s2;
                            for (int q = 0; q < 4; q++) { dn[q] = cand[id[q]]; w[q] = lam[q]; }
                        }
                    } else if (!have_in && sc > best_out) {
                        best_out = sc;
                        for (int q = 0; q < 4; q++) { dn[q] = cand[id[q]]; w[q] = lam[q]; }
                    }
                }
}

// Hole cut: one thread per element; background field cells whose centroid
// passes hole_test become holes (iblank 0).
__global__ void k_hole_cut(DMesh M, const int* block, hp_ov::HoleView H, int32_t* iblank, int* nholes) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (e > M.neles) return;
    int ib = row(M, e)[8];
    if (block[e - 1] == 0 && ib == 1) {
        double p[3];
        centroid(M, e, p);
        if (hp_ov::hole_test(H, p)) { ib = 0; atomicAdd(nholes, 1); }
    }
    iblank[e - 1] = ib;
}

// Device buffers of one build, freed on every exit.
struct Buffers {
    std::vector<void*> p;
    ~Buffers() {
        for (void* q : p) cudaFree(q);
    }
    template <class T>
    cudaError_t get(T** out, size_t n) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
        if (e == cudaSuccess) p.push_back(q);
        *out = (T*)q;
        return e;
    }
};

unsigned blocks_for(long long n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

#define OV_CUDA(call)                                         \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) { rc = HP_E_CUDA; goto done; } \
    } while (0)

// See include/hydraphase.h.
extern "C" int hp_overset_build_gpu(const hp_mesh* mesh, const int32_t* block, int32_t layers, int32_t outer_type,
                                    int32_t* iblank_out, hp_overset* out) {
    if (!out) return HP_E_ARG;
    std::memset(out, 0, sizeof *out);
    hp_ov::Prep P;
    int rc = hp_ov::prepare(mesh, block, layers, outer_type, iblank_out, P);
    if (rc != HP_OK) return rc;
    const int neles = mesh->neles, nodes = mesh->nodes, nf = (int)P.fr.size();
    out->nfringe = nf;
    out->fringe = (int32_t*)std::malloc(sizeof(int32_t) * (size_t)(nf + 1));
    out->donor = (int32_t*)std::malloc(sizeof(int32_t) * 4 * (size_t)(nf + 1));
    out->weight = (double*)std::malloc(sizeof(double) * 4 * (size_t)(nf + 1));
    if (!out->fringe || !out->donor || !out->weight) { hp_free_overset(out); return HP_E_NOMEM; }
    for (int f = 0; f < nf; f++) out->fringe[f] = P.fr[f];
    if (nf == 0) return HP_OK;
    {
        Buffers buf;
        cudaStream_t st = nullptr;
        double *x = nullptr, *y = nullptr, *z = nullptr, *w = nullptr;
        int32_t *elem = nullptr, *dn = nullptr;
        int *blk = nullptr, *ib = nullptr, *fr = nullptr, *donor = nullptr, *miss = nullptr;
        int* field[2] = {nullptr, nullptr};
        int *start[2] = {nullptr, nullptr}, *items[2] = {nullptr, nullptr};
        std::vector<int> hdonor(nf), hmiss;
        Bins bins[2];
        DMesh M;
        OV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        OV_CUDA(buf.get(&x, nodes));
        OV_CUDA(buf.get(&y, nodes));
        OV_CUDA(buf.get(&z, nodes));
        OV_CUDA(buf.get(&elem, 9 * (size_t)neles));
        OV_CUDA(buf.get(&blk, neles));
        OV_CUDA(buf.get(&ib, neles));
        OV_CUDA(buf.get(&fr, nf));
        OV_CUDA(buf.get(&donor, nf));
        OV_CUDA(buf.get(&miss, nf));
        OV_CUDA(buf.get(&dn, 4 * (size_t)nf));
        OV_CUDA(buf.get(&w, 4 * (size_t)nf));
        OV_CUDA(cudaMemcpyAsync(x, mesh->x, nodes * sizeof(double), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(y, mesh->y, nodes * sizeof(double), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(z, mesh->z, nodes * sizeof(double), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(elem, mesh->elem, 9 * (size_t)neles * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(blk, block, neles * sizeof(int), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(ib, iblank_out, neles * sizeof(int), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(fr, P.fr.data(), nf * sizeof(int), cudaMemcpyHostToDevice, st));
        M = DMesh{x, y, z, elem, neles};
        for (int b = 0; b < 2; b++) {
            const int n = (int)P.field[b].size();
            bins[b].g = P.grid[b];
            bins[b].nfield = n;
            bins[b].start = nullptr;
            bins[b].items = nullptr;
            if (n == 0) continue;
            const hp_ov::GridParams& g = P.grid[b];
            const size_t ncell = (size_t)g.n[0] * g.n[1] * g.n[2];
            int *cnt = nullptr, *fill = nullptr;
            OV_CUDA(buf.get(&field[b], n));
            OV_CUDA(cudaMemcpyAsync(field[b], P.field[b].data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
            OV_CUDA(buf.get(&cnt, ncell + 1));
            OV_CUDA(buf.get(&start[b], ncell + 1));
            OV_CUDA(buf.get(&fill, ncell));
            OV_CUDA(cudaMemsetAsync(cnt, 0, (ncell + 1) * sizeof(int), st));
            OV_CUDA(cudaMemsetAsync(fill, 0, ncell * sizeof(int), st));
            k_bin_count<<<blocks_for(n, 256), 256, 0, st>>>(M, g, field[b], n, cnt);
            OV_CUDA(cudaGetLastError());
            size_t tmp_bytes = 0;
            void* tmp = nullptr;
            OV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, start[b], (int)(ncell + 1), st));
            OV_CUDA(buf.get((char**)&tmp, tmp_bytes));
            OV_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, start[b], (int)(ncell + 1), st));
            int total = 0;
            OV_CUDA(cudaMemcpyAsync(&total, start[b] + ncell, sizeof(int), cudaMemcpyDeviceToHost, st));
            OV_CUDA(cudaStreamSynchronize(st));
            OV_CUDA(buf.get(&items[b], (size_t)total));
            k_bin_fill<<<blocks_for(n, 256), 256, 0, st>>>(M, g, field[b], n, start[b], fill, items[b]);
            OV_CUDA(cudaGetLastError());
            bins[b].start = start[b];
            bins[b].items = items[b];
        }
        k_donor<<<blocks_for(nf, 128), 128, 0, st>>>(M, blk, fr, nf, bins[0], bins[1], donor);
        OV_CUDA(cudaGetLastError());
        OV_CUDA(cudaMemcpyAsync(hdonor.data(), donor, nf * sizeof(int), cudaMemcpyDeviceToHost, st));
        OV_CUDA(cudaStreamSynchronize(st));
        // fringe cells inside no tet of the other block, which has field cells
        for (int f = 0; f < nf; f++) {
            const int B = 1 - block[P.fr[f] - 1];
            if (hdonor[f] == 0) {
                out->nfallback++;
                if (!P.field[B].empty()) hmiss.push_back(f);
            }
        }
        if (!hmiss.empty()) {
            OV_CUDA(cudaMemcpyAsync(miss, hmiss.data(), hmiss.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            k_nearest<<<(unsigned)hmiss.size(), 256, 0, st>>>(M, blk, fr, miss, field[0], (int)P.field[0].size(),
                                                              field[1], (int)P.field[1].size(), donor);
            OV_CUDA(cudaGetLastError());
        }
        k_weights<<<blocks_for(nf, 64), 64, 0, st>>>(M, blk, ib, fr, nf, donor, dn, w);
        OV_CUDA(cudaGetLastError());
        OV_CUDA(cudaMemcpyAsync(out->donor, dn, 4 * (size_t)nf * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        OV_CUDA(cudaMemcpyAsync(out->weight, w, 4 * (size_t)nf * sizeof(double), cudaMemcpyDeviceToHost, st));
        OV_CUDA(cudaStreamSynchronize(st));
    done:
        if (st) cudaStreamDestroy(st);
    }
    if (rc != HP_OK) hp_free_overset(out);
    return rc;
}

// See include/hydraphase.h.
extern "C" int hp_overset_hole_cut_gpu(const hp_mesh* mesh, const int32_t* block, int32_t wall_type, double margin,
                                       int32_t* iblank_out, int32_t* nholes) {
    if (!iblank_out) return HP_E_ARG;
    hp_ov::HolePrep HP;
    int rc = hp_ov::prepare_hole(mesh, block, wall_type, margin, HP);
    if (rc != HP_OK) return rc;
    const int neles = mesh->neles, nodes = mesh->nodes;
    {
        Buffers buf;
        cudaStream_t st = nullptr;
        double *x = nullptr, *y = nullptr, *z = nullptr, *tri = nullptr;
        int32_t *elem = nullptr, *ib = nullptr;
        int *blk = nullptr, *s3 = nullptr, *i3 = nullptr, *s2 = nullptr, *i2 = nullptr, *cnt = nullptr;
        int hcount = 0;
        hp_ov::HoleView V = HP.v;
        OV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        OV_CUDA(buf.get(&x, nodes));
        OV_CUDA(buf.get(&y, nodes));
        OV_CUDA(buf.get(&z, nodes));
        OV_CUDA(buf.get(&elem, 9 * (size_t)neles));
        OV_CUDA(buf.get(&blk, neles));
        OV_CUDA(buf.get(&ib, neles));
        OV_CUDA(buf.get(&cnt, 1));
        OV_CUDA(buf.get(&tri, HP.tri.size()));
        OV_CUDA(buf.get(&s3, HP.start3.size()));
        OV_CUDA(buf.get(&i3, HP.items3.size()));
        OV_CUDA(buf.get(&s2, HP.start2.size()));
        OV_CUDA(buf.get(&i2, HP.items2.size()));
        OV_CUDA(cudaMemcpyAsync(x, mesh->x, nodes * sizeof(double), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(y, mesh->y, nodes * sizeof(double), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(z, mesh->z, nodes * sizeof(double), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(elem, mesh->elem, 9 * (size_t)neles * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(blk, block, neles * sizeof(int), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(tri, HP.tri.data(), HP.tri.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(s3, HP.start3.data(), HP.start3.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(i3, HP.items3.data(), HP.items3.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(s2, HP.start2.data(), HP.start2.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemcpyAsync(i2, HP.items2.data(), HP.items2.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        OV_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), st));
        V.tri = tri;
        V.start3 = s3; V.items3 = i3;
        V.start2 = s2; V.items2 = i2;
        k_hole_cut<<<blocks_for(neles, 128), 128, 0, st>>>(DMesh{x, y, z, elem, neles}, blk, V, ib, cnt);
        OV_CUDA(cudaGetLastError());
        OV_CUDA(cudaMemcpyAsync(iblank_out, ib, neles * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        OV_CUDA(cudaMemcpyAsync(&hcount, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
        OV_CUDA(cudaStreamSynchronize(st));
        if (nholes) *nholes = hcount;
    done:
        if (st) cudaStreamDestroy(st);
    }
    return rc;
}
