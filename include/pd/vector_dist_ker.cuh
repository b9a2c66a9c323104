// vector_dist_ker.cuh -- device-side API for user kernels over libpdgpu.so views:
// the kernel half of OpenFPM pdata's vector_dist GPU interface.
//
// The reference's extension point is a user __global__ kernel that receives
// vd.toKernel() and cl.toKernel() by value and walks neighbours itself:
//
//   template<typename T, typename CL>
//   __global__ void k(pd::vector_dist_ker<3, T, pd::aggregate<T, T[3], T[3]>> vd, CL cl) {
//       size_t p = GET_PARTICLE(vd);                 // or: size_t p; GET_PARTICLE_SORT(p, cl);
//       pd::Point<3, T> xp = vd.getPos(p);
//       auto it = cl.getNNIteratorBox(cl.getCell(xp));
//       while (it.isNext()) {
//           auto q = it.get();                       // or it.get_sort() on a reordered vector
//           ... vd.template getProp<0>(q) ...
//           ++it;
//       }
//       vd.template getProp<1>(p)[0] = ...;
//   }
//   auto it = vd.getDomainIteratorGPU(32);
//   k<float, pd::CellList_gpu_ker<3, float>><<<it.wthr[0], it.thr[0]>>>(vd.toKernel(), cl.toKernel());
//
// Reference interfaces restated here (openfpm_pdata paths):
//   GET_PARTICLE, GET_PARTICLE_SORT          Vector/vector_dist_kernel.hpp:15-21
//   vector_dist_ker::getPos / getProp /
//     size_local / size                      Vector/vector_dist_kernel.hpp:57-305
//   CellList kernel view getCell /
//     getNNIteratorBox / get / get_sort /
//     getDomainSortIds / getGhostMarker      used at Vector/cuda/vector_dist_gpu_unit_tests.cu:54-113
//                                            (the class lives in openfpm_data, not in this tree)
//
// Conventions of this library, shared with its own kernels and the oracle:
//   * positions are 4-component records (x, y, z, unused) of the vector's type,
//     properties component-major with the vector's capacity as the stride;
//   * cell of x: ik = clamp(floor((x_k - lo_k) / spacing_k) + pad, 0, gs_k - 1) in
//     the position type (IEEE division), c = i0 + gs0 * (i1 + gs1 * i2);
//   * the box walk visits dz, dy, dx in [-nn_box, nn_box] with dx fastest and, in
//     each cell, the sorted slots in ascending order (ascending particle index,
//     real particles before ghosts); cells outside the padded grid are skipped;
//   * get() is the particle index in the vector's original order, get_sort() the
//     slot in cell order (the order of a vector reordered by updateCellListGPU
//     with PD_CL_GPU_REORDER until restoreOrder).
// Views are non-owning and invalid after any call that can reallocate the vector
// (map, ghost_get, resize) or rebuild the cell list; take them again afterwards.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <type_traits>

#include "../pdgpu.h"

namespace pd {

// ---------------------------------------------------------------------------
// Point<3,T>: the subset of openfpm_data's Point used inside kernels

template <unsigned int dim, typename T> struct Point {
    static_assert(dim == 3, "this library's particles are three-dimensional");
    T v[3];
    Point() = default;
    __host__ __device__ Point(T x, T y, T z) : v{x, y, z} {}
    __host__ __device__ T& operator[](int i) { return v[i]; }
    __host__ __device__ const T& operator[](int i) const { return v[i]; }
    __host__ __device__ T get(int i) const { return v[i]; }
    __host__ __device__ T norm() const { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
    __host__ __device__ Point& operator+=(const Point& o) {
        for (int i = 0; i < 3; ++i) v[i] += o.v[i];
        return *this;
    }
    __host__ __device__ Point& operator-=(const Point& o) {
        for (int i = 0; i < 3; ++i) v[i] -= o.v[i];
        return *this;
    }
    __host__ __device__ Point& operator*=(T s) {
        for (int i = 0; i < 3; ++i) v[i] *= s;
        return *this;
    }
    __host__ __device__ Point& operator/=(T s) {
        for (int i = 0; i < 3; ++i) v[i] /= s;
        return *this;
    }
    __host__ __device__ friend Point operator+(Point a, const Point& b) { return a += b; }
    __host__ __device__ friend Point operator-(Point a, const Point& b) { return a -= b; }
    __host__ __device__ friend Point operator*(T s, Point a) { return a *= s; }
    __host__ __device__ friend Point operator*(Point a, T s) { return a *= s; }
};

// ---------------------------------------------------------------------------
// property list and accessors

template <typename... Props> struct aggregate {
    static constexpr int max_prop = (int)sizeof...(Props);
};

namespace detail {
template <int k, typename... Ps> struct nth;
template <typename P, typename... Ps> struct nth<0, P, Ps...> { typedef P type; };
template <int k, typename P, typename... Ps> struct nth<k, P, Ps...> { typedef typename nth<k - 1, Ps...>::type type; };

template <typename S> struct pd_type;
template <> struct pd_type<float> { static constexpr int value = PD_F32; };
template <> struct pd_type<double> { static constexpr int value = PD_F64; };
template <> struct pd_type<int> { static constexpr int value = PD_I32; };
template <> struct pd_type<unsigned int> { static constexpr int value = PD_U32; };
template <> struct pd_type<long long> { static constexpr int value = PD_I64; };

// component c of particle p of an array property lives at base[c * stride + p]
template <typename S> struct comp_ref {
    S* base;
    long stride;
    __device__ S& operator[](int c) const { return base[(long)c * stride]; }
};

template <typename P> struct prop_info {  // scalar property
    typedef P scalar;
    static constexpr int ncomp = 1;
    typedef P& ref;
    __device__ static ref at(void* col, long stride, long p) {
        (void)stride;
        return static_cast<P*>(col)[p];
    }
};
template <typename S, int N> struct prop_info<S[N]> {  // array property S[N]
    typedef S scalar;
    static constexpr int ncomp = N;
    typedef comp_ref<S> ref;
    __device__ static ref at(void* col, long stride, long p) { return ref{static_cast<S*>(col) + p, stride}; }
};

template <typename T> struct rec4;
template <> struct rec4<float> { typedef float4 type; };
template <> struct rec4<double> { typedef double4 type; };
}  // namespace detail

// position record of particle p: pos[k] reads and writes coordinate k; converts to Point
template <typename T> struct pos_ref {
    T* r;
    __device__ T& operator[](int k) const { return r[k]; }
    __device__ operator Point<3, T>() const { return Point<3, T>(r[0], r[1], r[2]); }
};

template <unsigned int dim, typename St, typename Agg> struct vector_dist_ker;

// vector_dist_ker<3, St, aggregate<Props...>>: by-value device view of a vector
template <typename St, typename... Props> struct vector_dist_ker<3, St, aggregate<Props...>> {
    static_assert(std::is_same<St, float>::value || std::is_same<St, double>::value, "St must be float or double");
    static constexpr int n_props = (int)sizeof...(Props);
    typedef St stype;

    St* pos_;
    void* prop_[n_props > 0 ? n_props : 1];
    long stride_, size_local_, size_;

    vector_dist_ker() = default;
    // from toKernel() (pd_view_t): the property list must match the vector's
    __host__ vector_dist_ker(const pd_view_t& v) {
        const int want = detail::pd_type<St>::value;
        if (v.dtype != want) throw std::runtime_error("vector_dist_ker: position type differs from the vector's");
        if (v.n_prop < n_props) throw std::runtime_error("vector_dist_ker: the vector has fewer properties");
        check_props<0, Props...>(v);
        pos_ = static_cast<St*>(v.pos);
        for (int k = 0; k < n_props; ++k) prop_[k] = v.prop[k];
        stride_ = v.stride;
        size_local_ = v.size_local;
        size_ = v.size;
    }

    __device__ long size_local() const { return size_local_; }
    __device__ long size() const { return size_; }

    // vd.getPos(p)[k] (read and write); Point<3,St> xp = vd.getPos(p)
    __device__ pos_ref<St> getPos(long p) const { return pos_ref<St>{pos_ + 4 * p}; }

    // vd.template getProp<k>(p): St& for a scalar property, [c] for an array property
    template <int k>
    __device__ typename detail::prop_info<typename detail::nth<k, Props...>::type>::ref getProp(long p) const {
        typedef detail::prop_info<typename detail::nth<k, Props...>::type> I;
        return I::at(prop_[k], stride_, p);
    }

  private:
    template <int k> __host__ static void check_props(const pd_view_t&) {}
    template <int k, typename P, typename... Rest> __host__ static void check_props(const pd_view_t& v) {
        typedef detail::prop_info<P> I;
        if (v.prop_type[k] != detail::pd_type<typename I::scalar>::value || v.prop_ncomp[k] != I::ncomp)
            throw std::runtime_error("vector_dist_ker: property " + std::to_string(k) +
                                     " differs in type or components from the vector's");
        check_props<k + 1, Rest...>(v);
    }
};

// ---------------------------------------------------------------------------
// cell list

template <unsigned int dim, typename T> struct CellList_gpu_ker;

// box walk of (2 nn_box + 1)^3 cells around a cell
template <typename T> struct NNIteratorBox {
    const int* cs;
    const int* sorted;
    int gs0, gs1, gs2, r;
    int c0, c1, c2;  // centre cell coordinates
    int dx, dy, dz;
    int k, ke;  // current slot and end of the current cell

    __device__ bool isNext() const { return k < ke; }
    __device__ int get() const { return sorted[k]; }
    __device__ int get_sort() const { return k; }
    __device__ NNIteratorBox& operator++() {
        ++k;
        if (k >= ke) next_cell();
        return *this;
    }
    // position on the first slot of the next non-empty cell of the box; k = ke = 0 at the end
    __device__ void next_cell() {
        for (;;) {
            if (++dx > r) {
                dx = -r;
                if (++dy > r) {
                    dy = -r;
                    if (++dz > r) {
                        k = ke = 0;
                        return;
                    }
                }
            }
            if (enter()) return;
        }
    }
    // the cell (c + d) when it lies in the grid and is non-empty
    __device__ bool enter() {
        const int x = c0 + dx, y = c1 + dy, z = c2 + dz;
        if (x < 0 || y < 0 || z < 0 || x >= gs0 || y >= gs1 || z >= gs2) return false;
        const long c = x + (long)gs0 * (y + (long)gs1 * z);
        k = cs[c];
        ke = cs[c + 1];
        return k < ke;
    }
};

// getDomainSortIds().template get<0>(t): sorted slot of the t-th domain particle
struct dom_sort_ids {
    const int* ids;
    template <int> __device__ int get(long t) const { return ids[t]; }
};

template <typename T> struct CellList_gpu_ker<3, T> {
    const int* cell_start_;
    const int* sorted_;
    const int* dom_sort_;
    int gs_[3];
    int pad_, nn_box_;
    T lo_[3], sp_[3];
    long ghost_marker_;

    CellList_gpu_ker() = default;
    // from CellList_gpu::toKernel() (pd_cl_view_t)
    __host__ CellList_gpu_ker(const pd_cl_view_t& v) {
        cell_start_ = v.cell_start;
        sorted_ = v.sorted_ids;
        dom_sort_ = v.dom_sort_ids;
        for (int d = 0; d < 3; ++d) {
            gs_[d] = v.gs[d];
            lo_[d] = (T)v.box_lo[d];
            sp_[d] = (T)v.spacing[d];
        }
        pad_ = v.pad;
        nn_box_ = v.nn_box;
        ghost_marker_ = v.ghost_marker;
    }

    // cell index of a position (clamped into the padded grid, as the build does)
    __device__ int getCell(const Point<3, T>& x) const {
        int i[3];
        for (int d = 0; d < 3; ++d) {
            const T q = floor((x[d] - lo_[d]) / sp_[d]);
            int c = (q > T(-1e9) && q < T(1e9)) ? (int)q + pad_ : 0;
            c = c < 0 ? 0 : (c > gs_[d] - 1 ? gs_[d] - 1 : c);
            i[d] = c;
        }
        return i[0] + gs_[0] * (i[1] + gs_[1] * i[2]);
    }

    __device__ NNIteratorBox<T> getNNIteratorBox(int cell) const {
        NNIteratorBox<T> it;
        it.cs = cell_start_;
        it.sorted = sorted_;
        it.gs0 = gs_[0];
        it.gs1 = gs_[1];
        it.gs2 = gs_[2];
        it.r = nn_box_;
        it.c0 = cell % gs_[0];
        it.c1 = (cell / gs_[0]) % gs_[1];
        it.c2 = cell / (gs_[0] * gs_[1]);
        it.dx = it.dy = it.dz = -nn_box_;
        if (!it.enter()) it.next_cell();
        return it;
    }

    __device__ long getGhostMarker() const { return ghost_marker_; }
    __device__ dom_sort_ids getDomainSortIds() const { return dom_sort_ids{dom_sort_}; }
};

}  // namespace pd

// Thread-to-particle macros of the reference (Vector/vector_dist_kernel.hpp:15-17).
// GET_PARTICLE(vd): this thread's domain particle, or return past size_local().
#ifndef GET_PARTICLE
#define GET_PARTICLE(vd)                                                                  \
    blockDim.x * blockIdx.x + threadIdx.x;                                                \
    if (blockDim.x * blockIdx.x + threadIdx.x >= static_cast<unsigned int>((vd).size_local())) { \
        return;                                                                           \
    }
#endif
// GET_PARTICLE_SORT(p, cl): the sorted slot of this thread's domain particle, or return.
#ifndef GET_PARTICLE_SORT
#define GET_PARTICLE_SORT(p, NN)                                                          \
    if (blockDim.x * blockIdx.x + threadIdx.x >= (NN).getGhostMarker()) {                 \
        return;                                                                           \
    } else {                                                                              \
        p = (NN).getDomainSortIds().template get<0>(blockDim.x * blockIdx.x + threadIdx.x); \
    }
#endif
