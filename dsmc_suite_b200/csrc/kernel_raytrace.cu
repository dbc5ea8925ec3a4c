// kernel_raytrace.cu - Monte Carlo shadow flux of a body mesh on the GPU (the reference's
// src/raytracer/shadow_maker.c:198-238, which traces with Intel Embree on the CPU).
//
// For rotation phase t and face f: the sun direction s(t) = (cos(-za) sin(phi), cos(-za) cos(phi),
// sin(-za)) with phi = 2 pi (t + 1/2) / tt + pi; faces turned away (s . n < 0) get 0; otherwise
// Nmonte points of the face are drawn with rand_r from the seed t * nface + f + 42 (the
// reference's sequence), each lifted 1e-3 along the face normal and tested for any hit along s,
// and the face gets (1 - shadowed / Nmonte) (s . n).
//
// GPU design: one thread per (phase, face), consecutive threads on consecutive faces at one phase
// (rays of a warp start close together and share the direction, so their BVH walks are coherent).
// The BVH is built on the host (binned surface-area heuristic, at most 4 triangles per leaf,
// median splits below depth 40 so that every path fits the 64-entry traversal stack) and walked
// for any hit; triangles are stored as (v0, e1, e2) float4 triples for the Moller-Trumbore test.
// Compiled with -fmad=false so that the sample points and the flux factor follow the reference's
// FP64 operation order; the ray itself is FP32 like Embree's.
#include "dsmc_kernels.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

namespace dsmc {
namespace {

struct BvhNode {
    float lo[3];
    int first;      // inner node: index of the left child (right = first + 1); leaf: first triangle
    float hi[3];
    int count;      // 0 = inner node, else triangles in the leaf
};

constexpr int kLeaf = 4;
constexpr int kStack = 64;
constexpr int kMedianDepth = 40;

struct Builder {
    const std::vector<float> &V;   // [npoint][3]
    const int *F;                  // [nface][3]
    int nface;
    std::vector<int> idx;
    std::vector<float> cen, blo, bhi;   // per triangle centroid and box
    std::vector<BvhNode> nodes;
    std::atomic<int> used{0};      // nodes handed out (subtrees are built by parallel threads)

    Builder(const std::vector<float> &v, const int *f, int n) : V(v), F(f), nface(n) {
        idx.resize(n);
        cen.resize(3 * static_cast<size_t>(n));
        blo.resize(3 * static_cast<size_t>(n));
        bhi.resize(3 * static_cast<size_t>(n));
        for (int k = 0; k < n; k++) {
            idx[k] = k;
            for (int a = 0; a < 3; a++) {
                float lo = 1e38f, hi = -1e38f;
                for (int j = 0; j < 3; j++) {
                    const float x = V[3 * static_cast<size_t>(F[3 * k + j]) + a];
                    lo = std::min(lo, x);
                    hi = std::max(hi, x);
                }
                blo[3 * k + a] = lo;
                bhi[3 * k + a] = hi;
                cen[3 * k + a] = 0.5f * (lo + hi);
            }
        }
    }

    static float area(const float lo[3], const float hi[3]) {
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return dx < 0 ? 0.0f : 2.0f * (dx * dy + dy * dz + dz * dx);
    }

    void box_of(int b, int e, float lo[3], float hi[3]) const {
        for (int a = 0; a < 3; a++) { lo[a] = 1e38f; hi[a] = -1e38f; }
        for (int k = b; k < e; k++)
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], blo[3 * idx[k] + a]);
                hi[a] = std::max(hi[a], bhi[3 * idx[k] + a]);
            }
    }

    void build() {
        nodes.assign(2 * static_cast<size_t>(nface) + 1, BvhNode{});
        used = 1;
        split(0, 0, nface, 0);
        nodes.resize(static_cast<size_t>(used.load()));
    }

    void split(int node, int b, int e, int depth) {
        float lo[3], hi[3];
        box_of(b, e, lo, hi);
        for (int a = 0; a < 3; a++) { nodes[node].lo[a] = lo[a]; nodes[node].hi[a] = hi[a]; }
        if (e - b <= kLeaf) { nodes[node].first = b; nodes[node].count = e - b; return; }
        float clo[3] = {1e38f, 1e38f, 1e38f}, chi[3] = {-1e38f, -1e38f, -1e38f};
        for (int k = b; k < e; k++)
            for (int a = 0; a < 3; a++) {
                clo[a] = std::min(clo[a], cen[3 * idx[k] + a]);
                chi[a] = std::max(chi[a], cen[3 * idx[k] + a]);
            }
        int axis = 0;
        for (int a = 1; a < 3; a++)
            if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
        const float ext = chi[axis] - clo[axis];
        if (!(ext > 0.0f)) { nodes[node].first = b; nodes[node].count = e - b; return; }   // coincident
        int mid = -1;
        if (depth < kMedianDepth) {
            constexpr int kBins = 12;
            int cnt[kBins] = {0};
            float bl[kBins][3], bh[kBins][3];
            for (int i = 0; i < kBins; i++)
                for (int a = 0; a < 3; a++) { bl[i][a] = 1e38f; bh[i][a] = -1e38f; }
            auto bin_of = [&](int t) {
                const int i = static_cast<int>((cen[3 * t + axis] - clo[axis]) / ext * kBins);
                return std::min(std::max(i, 0), kBins - 1);
            };
            for (int k = b; k < e; k++) {
                const int t = idx[k], i = bin_of(t);
                cnt[i]++;
                for (int a = 0; a < 3; a++) {
                    bl[i][a] = std::min(bl[i][a], blo[3 * t + a]);
                    bh[i][a] = std::max(bh[i][a], bhi[3 * t + a]);
                }
            }
            float best = 1e38f;
            int best_i = -1;
            for (int s = 1; s < kBins; s++) {
                float l0[3] = {1e38f, 1e38f, 1e38f}, l1[3] = {-1e38f, -1e38f, -1e38f};
                float r0[3] = {1e38f, 1e38f, 1e38f}, r1[3] = {-1e38f, -1e38f, -1e38f};
                int nl = 0, nr = 0;
                for (int i = 0; i < kBins; i++) {
                    float *o0 = i < s ? l0 : r0, *o1 = i < s ? l1 : r1;
                    (i < s ? nl : nr) += cnt[i];
                    for (int a = 0; a < 3; a++) { o0[a] = std::min(o0[a], bl[i][a]); o1[a] = std::max(o1[a], bh[i][a]); }
                }
                if (!nl || !nr) continue;
                const float cost = nl * area(l0, l1) + nr * area(r0, r1);
                if (cost < best) { best = cost; best_i = s; }
            }
            if (best_i > 0) {
                int *p = std::partition(idx.data() + b, idx.data() + e, [&](int t) { return bin_of(t) < best_i; });
                mid = static_cast<int>(p - idx.data());
            }
        }
        if (mid <= b || mid >= e) {   // median split along the axis
            mid = (b + e) / 2;
            std::nth_element(idx.data() + b, idx.data() + mid, idx.data() + e,
                             [&](int x, int y) { return cen[3 * x + axis] < cen[3 * y + axis]; });
        }
        const int left = used.fetch_add(2);
        nodes[node].first = left;
        nodes[node].count = 0;
        // the two subtrees touch disjoint index ranges and nodes: the upper levels of a large
        // mesh are split across threads (at most 8)
        if (depth < 3 && e - b > 20000) {
            std::thread t([&] { split(left, b, mid, depth + 1); });
            split(left + 1, mid, e, depth + 1);
            t.join();
        } else {
            split(left, b, mid, depth + 1);
            split(left + 1, mid, e, depth + 1);
        }
    }
};

// glibc's rand_r: three steps of the ANSI C linear congruential generator, 11 + 10 + 10 bits.
__device__ __forceinline__ int rand_r_dev(unsigned int *seed) {
    unsigned int next = *seed;
    next = next * 1103515245u + 12345u;
    int result = static_cast<int>((next / 65536u) % 2048u);
    next = next * 1103515245u + 12345u;
    result = (result << 10) ^ static_cast<int>((next / 65536u) % 1024u);
    next = next * 1103515245u + 12345u;
    result = (result << 10) ^ static_cast<int>((next / 65536u) % 1024u);
    *seed = next;
    return result;
}

struct ShadowArgs {
    const BvhNode *nodes;
    const float4 *tris;     // [ntri][3]: v0, e1 = v1 - v0, e2 = v2 - v0 (BVH order)
    int nnodes;
    const int *facet;       // [nface][3], 0-based
    const double *spot;     // [npoint][3]
    const double *normal;   // [nface][3]
    int nface, tt, nmonte;
    double za;
    double *F;              // [nface][tt]
    int *overflow;          // traversal stack overflows (0 by construction of the tree)
};

__device__ bool slab(const BvhNode &n, const float o[3], const float inv[3], float tmax) {
    float t0 = 0.0f, t1 = tmax;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float ta = (n.lo[a] - o[a]) * inv[a], tb = (n.hi[a] - o[a]) * inv[a];
        if (ta > tb) { const float x = ta; ta = tb; tb = x; }
        t0 = fmaxf(t0, ta);
        t1 = fminf(t1, tb);
    }
    return t0 <= t1;
}

// Moller-Trumbore with the ray parameter in [0, tmax] (Embree's tnear = 0, tfar = 1e30).
__device__ bool hit_triangle(const float4 *t, const float o[3], const float d[3], float tmax) {
    const float4 v0 = t[0], e1 = t[1], e2 = t[2];
    const float px = d[1] * e2.z - d[2] * e2.y, py = d[2] * e2.x - d[0] * e2.z, pz = d[0] * e2.y - d[1] * e2.x;
    const float det = e1.x * px + e1.y * py + e1.z * pz;
    if (det == 0.0f) return false;
    const float inv = 1.0f / det;
    const float sx = o[0] - v0.x, sy = o[1] - v0.y, sz = o[2] - v0.z;
    const float u = (sx * px + sy * py + sz * pz) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    const float qx = sy * e1.z - sz * e1.y, qy = sz * e1.x - sx * e1.z, qz = sx * e1.y - sy * e1.x;
    const float v = (d[0] * qx + d[1] * qy + d[2] * qz) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    const float tt = (e2.x * qx + e2.y * qy + e2.z * qz) * inv;
    return tt >= 0.0f && tt <= tmax;
}

__device__ bool occluded(const ShadowArgs &a, const float o[3], const float d[3]) {
    const float tmax = 1e30f;
    float inv[3];
#pragma unroll
    for (int k = 0; k < 3; k++) inv[k] = 1.0f / (d[k] != 0.0f ? d[k] : 1e-30f);
    int stack[kStack];
    int sp = 0, n = 0;
    for (int it = 0; it < 2 * a.nnodes + 2; it++) {
        const BvhNode nd = a.nodes[n];
        bool descend = false;
        if (slab(nd, o, inv, tmax)) {
            if (nd.count > 0) {
                for (int k = nd.first; k < nd.first + nd.count; k++)
                    if (hit_triangle(a.tris + 3 * k, o, d, tmax)) return true;
            } else if (sp < kStack) {
                stack[sp++] = nd.first + 1;
                n = nd.first;
                descend = true;
            } else {
                atomicAdd(a.overflow, 1);
            }
        }
        if (!descend) {
            if (sp == 0) return false;
            n = stack[--sp];
        }
    }
    return false;
}

__global__ void shadow_kernel(const ShadowArgs a) {
    const long long g = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= static_cast<long long>(a.nface) * a.tt) return;
    const int t = static_cast<int>(g / a.nface), nf = static_cast<int>(g % a.nface);
    constexpr double kPi = 3.14159265358979323846;
    const double fi = ((t + 0.5) / a.tt) * 2.0 * kPi + kPi;
    const double sun[3] = {cos(-a.za) * sin(fi), cos(-a.za) * cos(fi), sin(-a.za)};
    const double *fn = a.normal + 3 * nf;
    const double c6 = sun[0] * fn[0] + sun[1] * fn[1] + sun[2] * fn[2];
    double *out = a.F + static_cast<long long>(nf) * a.tt + t;
    if (c6 < 0) { *out = 0.0; return; }
    const double *A = a.spot + 3 * a.facet[3 * nf], *B = a.spot + 3 * a.facet[3 * nf + 1],
                 *C = a.spot + 3 * a.facet[3 * nf + 2];
    const float d[3] = {static_cast<float>(sun[0]), static_cast<float>(sun[1]), static_cast<float>(sun[2])};
    const double eps = static_cast<double>(1e-3f);   // the reference's float offset, promoted
    unsigned int seed = static_cast<unsigned int>(t * a.nface + nf + 42);
    int shadowed = 0;
    for (int mc = 0; mc < a.nmonte; mc++) {
        const double r1 = sqrt(static_cast<double>(rand_r_dev(&seed)) / 2147483647.0);
        const double r2 = static_cast<double>(rand_r_dev(&seed)) / 2147483647.0;
        const double wa = 1.0 - r1, wb = r1 * (1.0 - r2), wc = r1 * r2;
        float o[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double p = A[k] * wa + B[k] * wb + C[k] * wc;
            o[k] = static_cast<float>(p + eps * fn[k]);
        }
        if (occluded(a, o, d)) shadowed++;
    }
    *out = (1.0 - static_cast<double>(shadowed) / a.nmonte) * c6;
}

}  // namespace

cudaError_t shadow_flux(int npoint, const double *spot, int nface, const int *facet,
                        const double *normal, double za, int tt, int nmonte, double *F_host,
                        cudaStream_t stream, long long *overflows, double *kernel_ms) {
    std::vector<float> V(3 * static_cast<size_t>(npoint));
    for (size_t k = 0; k < V.size(); k++) V[k] = static_cast<float>(spot[k]);
    Builder bld(V, facet, nface);
    bld.build();
    std::vector<float4> tris(3 * static_cast<size_t>(nface));
    for (int k = 0; k < nface; k++) {
        const int f = bld.idx[k];
        const float *v0 = &V[3 * static_cast<size_t>(facet[3 * f])], *v1 = &V[3 * static_cast<size_t>(facet[3 * f + 1])],
                    *v2 = &V[3 * static_cast<size_t>(facet[3 * f + 2])];
        tris[3 * k + 0] = make_float4(v0[0], v0[1], v0[2], 0.0f);
        tris[3 * k + 1] = make_float4(v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2], 0.0f);
        tris[3 * k + 2] = make_float4(v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2], 0.0f);
    }
    struct Bufs {
        void *p[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        ~Bufs() { for (void *q : p) if (q) cudaFree(q); }
    } b;
    const size_t nn = bld.nodes.size(), nfc = static_cast<size_t>(nface), np = static_cast<size_t>(npoint);
    const size_t nF = nfc * static_cast<size_t>(tt);
    cudaError_t e;
    if ((e = cudaMalloc(&b.p[0], nn * sizeof(BvhNode))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&b.p[1], tris.size() * sizeof(float4))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&b.p[2], nfc * 3 * sizeof(int))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&b.p[3], np * 3 * sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&b.p[4], nfc * 3 * sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&b.p[5], nF * sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&b.p[6], sizeof(int))) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b.p[0], bld.nodes.data(), nn * sizeof(BvhNode), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b.p[1], tris.data(), tris.size() * sizeof(float4), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b.p[2], facet, nfc * 3 * sizeof(int), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b.p[3], spot, np * 3 * sizeof(double), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b.p[4], normal, nfc * 3 * sizeof(double), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(b.p[6], 0, sizeof(int), stream)) != cudaSuccess)
        return e;
    ShadowArgs a{};
    a.nodes = static_cast<const BvhNode *>(b.p[0]);
    a.tris = static_cast<const float4 *>(b.p[1]);
    a.nnodes = static_cast<int>(nn);
    a.facet = static_cast<const int *>(b.p[2]);
    a.spot = static_cast<const double *>(b.p[3]);
    a.normal = static_cast<const double *>(b.p[4]);
    a.nface = nface;
    a.tt = tt;
    a.nmonte = nmonte;
    a.za = za;
    a.F = static_cast<double *>(b.p[5]);
    a.overflow = static_cast<int *>(b.p[6]);
    const int block = 128;
    const long long threads = static_cast<long long>(nfc) * tt;
    struct Events {
        cudaEvent_t e[2] = {nullptr, nullptr};
        ~Events() { for (cudaEvent_t x : e) if (x) cudaEventDestroy(x); }
    } ev;
    if ((e = cudaEventCreate(&ev.e[0])) != cudaSuccess || (e = cudaEventCreate(&ev.e[1])) != cudaSuccess ||
        (e = cudaEventRecord(ev.e[0], stream)) != cudaSuccess)
        return e;
    shadow_kernel<<<static_cast<unsigned>((threads + block - 1) / block), block, 0, stream>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ev.e[1], stream)) != cudaSuccess) return e;
    int ovf = 0;
    if ((e = cudaMemcpyAsync(F_host, b.p[5], nF * sizeof(double), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&ovf, b.p[6], sizeof(int), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess)
        return e;
    if (overflows) *overflows = ovf;
    float ms = 0.f;
    if (kernel_ms && cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]) == cudaSuccess) *kernel_ms = ms;
    return cudaSuccess;
}

}  // namespace dsmc
