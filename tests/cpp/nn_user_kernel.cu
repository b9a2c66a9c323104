// A user program of the device-side API (include/pd/vector_dist_ker.cuh): user
// __global__ kernels written against vd.toKernel() / cl.toKernel(), launched with
// getDomainIteratorGPU, as the reference's GPU cell-list test does
// (Vector/cuda/vector_dist_gpu_unit_tests.cu:259-423).
//
// Reads n and n lines "x y z" (floats in the unit box) from stdin; runs
//   map, a property-initialising kernel, ghost_get<0>, getCellListGPU(0.1),
//   updateCellListGPU<0> (with PD_CL_GPU_REORDER when argv[1] is "sorted"),
//   the pair kernel (GET_PARTICLE + get(), or GET_PARTICLE_SORT + get_sort()),
//   restoreOrder<1> after the sorted variant;
// and prints "n_all <size with ghosts>", then one line "x y z p0" per particle
// (ghosts included) and one line "f0 f1 f2" per domain particle.
#include <cstdio>
#include <cstring>
#include <vector>

#include "pd/vector_dist_gpu.hpp"
#include "pd/vector_dist_ker.cuh"

typedef pd::aggregate<float, float[3], float[3]> props_t;

// prop0 = x + y + z, prop1 = (x + y, x + z, y + z)
template <typename T> __global__ void set_props(pd::vector_dist_ker<3, T, pd::aggregate<T, T[3], T[3]>> vd) {
    size_t p = GET_PARTICLE(vd);
    pd::Point<3, T> x = vd.getPos(p);
    vd.template getProp<0>(p) = x[0] + x[1] + x[2];
    vd.template getProp<1>(p)[0] = x[0] + x[1];
    vd.template getProp<1>(p)[1] = x[0] + x[2];
    vd.template getProp<1>(p)[2] = x[1] + x[2];
}

// sum over the box neighbours q != p of prop0(q) times the unit vector from p to q
template <typename T, typename CL>
__global__ void pair_sum(pd::vector_dist_ker<3, T, pd::aggregate<T, T[3], T[3]>> vd, CL cl) {
    size_t p = GET_PARTICLE(vd);
    const pd::Point<3, T> xp = vd.getPos(p);
    pd::Point<3, T> acc(0, 0, 0);
    for (auto it = cl.getNNIteratorBox(cl.getCell(xp)); it.isNext(); ++it) {
        const int q = it.get();
        if (q == (int)p) continue;
        pd::Point<3, T> d = pd::Point<3, T>(vd.getPos(q)) - xp;
        const T len = d.norm();
        if (len > T(1e-6)) {
            d /= len;
            acc += vd.template getProp<0>(q) * d;
        }
    }
    for (int k = 0; k < 3; ++k) vd.template getProp<1>(p)[k] = acc[k];
}

// the same sum on the reordered vector: threads take the sorted slots of the
// domain particles, neighbours are sorted slots
template <typename T, typename CL>
__global__ void pair_sum_sorted(pd::vector_dist_ker<3, T, pd::aggregate<T, T[3], T[3]>> vd, CL cl) {
    size_t p;
    GET_PARTICLE_SORT(p, cl);
    const pd::Point<3, T> xp = vd.getPos(p);
    pd::Point<3, T> acc(0, 0, 0);
    auto it = cl.getNNIteratorBox(cl.getCell(xp));
    while (it.isNext()) {
        const int q = it.get_sort();
        if (q != (int)p) {
            pd::Point<3, T> d = pd::Point<3, T>(vd.getPos(q)) - xp;
            const T len = d.norm();
            if (len > T(1e-6)) {
                d /= len;
                acc += vd.template getProp<0>(q) * d;
            }
        }
        ++it;
    }
    for (int k = 0; k < 3; ++k) vd.template getProp<1>(p)[k] = acc[k];
}

static int cuda_ok(const char* what) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        return 0;
    }
    return 1;
}

int main(int argc, char** argv) {
    const bool sorted = argc > 1 && strcmp(argv[1], "sorted") == 0;
    long n;
    if (scanf("%ld", &n) != 1) return 2;
    pd::vector_dist_gpu<float> vd(0, {0, 0, 0}, {1, 1, 1}, {PD_NON_PERIODIC, PD_NON_PERIODIC, PD_NON_PERIODIC},
                                  {0.1, 0.1, 0.1}, {{PD_F32, 1}, {PD_F32, 3}, {PD_F32, 3}});
    for (long i = 0; i < n; ++i) {
        vd.add();
        float* x = vd.getLastPos();
        if (scanf("%f %f %f", &x[0], &x[1], &x[2]) != 3) return 2;
    }
    vd.hostToDevicePos();
    vd.map();
    pd_launch_t it = vd.getDomainIteratorGPU(32);
    set_props<float><<<it.wthr[0], it.thr[0]>>>(vd.toKernel());
    if (!cuda_ok("set_props")) return 4;
    vd.ghost_get({0});
    pd::CellList_gpu cl = vd.getCellListGPU(0.1f, PD_CL_NON_SYMMETRIC | (sorted ? PD_CL_GPU_REORDER : 0));
    vd.updateCellListGPU(cl, {0});
    it = vd.getDomainIteratorGPU(32);
    typedef pd::CellList_gpu_ker<3, float> clk_t;
    if (sorted)
        pair_sum_sorted<float, clk_t><<<it.wthr[0], it.thr[0]>>>(vd.toKernel(), cl.toKernel());
    else
        pair_sum<float, clk_t><<<it.wthr[0], it.thr[0]>>>(vd.toKernel(), cl.toKernel());
    if (!cuda_ok("pair kernel")) return 4;
    if (sorted) vd.restoreOrder(cl, {1});
    vd.deviceToHostPos();
    vd.deviceToHostProp(0);
    vd.deviceToHostProp(1);
    const long n_all = vd.size_local_with_ghost(), n_dom = vd.size_local();
    printf("n_all %ld %ld\n", n_all, n_dom);
    for (long p = 0; p < n_all; ++p) {
        const float* x = vd.getPos(p);
        printf("%.9g %.9g %.9g %.9g\n", x[0], x[1], x[2], vd.getProp<float>(0, p));
    }
    for (long p = 0; p < n_dom; ++p)
        printf("%.9g %.9g %.9g\n", vd.getProp<float>(1, p, 0), vd.getProp<float>(1, p, 1), vd.getProp<float>(1, p, 2));
    return 0;
}
