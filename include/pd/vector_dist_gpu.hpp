// vector_dist_gpu.hpp -- header-only C++ host API over libpdgpu.so with the
// method names of OpenFPM pdata's vector_dist (Vector/vector_dist.hpp).
//
// A user of the reference's single-GPU particle path switches by replacing
//   vector_dist_gpu<3,St,aggregate<...>> vd(n, box, bc, ghost);
// with
//   pd::vector_dist_gpu<St> vd(n, lo, hi, bc, ghost, {{PD_F64,3}, ...});
// and keeps the calls: getPos/getProp (host mirror), add/getLastPos/getLastProp,
// hostToDevicePos/Prop,
// map, ghost_get, getCellListGPU/updateCellListGPU/restoreOrder,
// getVerlet/updateVerlet, getDomainIteratorGPU, toKernel.  Errors throw
// std::runtime_error with the library's message (the reference's
// ACTION_ON_ERROR under SE_CLASS1).  Host mirrors are std::vectors; every
// device transfer is explicit, as in the reference.
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../pdgpu.h"

namespace pd {

inline void check(int rc) {
    if (rc != PD_OK) throw std::runtime_error(std::string("libpdgpu: ") + pd_last_error());
}

struct prop_desc {
    int type;
    int ncomp;
};

inline int type_bytes(int t) { return (t == PD_F64 || t == PD_I64) ? 8 : 4; }

template <typename St> class vector_dist_gpu;

// CellList_gpu handle
class CellList_gpu {
    pd_cl h_ = nullptr;

  public:
    CellList_gpu() = default;
    explicit CellList_gpu(pd_cl h) : h_(h) {}
    CellList_gpu(const CellList_gpu&) = delete;
    CellList_gpu& operator=(const CellList_gpu&) = delete;
    CellList_gpu(CellList_gpu&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    CellList_gpu& operator=(CellList_gpu&& o) noexcept {
        std::swap(h_, o.h_);
        return *this;
    }
    ~CellList_gpu() {
        if (h_) pd_celllist_destroy(h_);
    }
    pd_cl handle() const { return h_; }
    pd_cl_view_t toKernel() const {
        pd_cl_view_t v;
        check(pd_celllist_view(h_, &v));
        return v;
    }
};

// VerletList handle (full list, self included)
class VerletList {
    pd_vl h_ = nullptr;
    long n_ = 0;

  public:
    VerletList() = default;
    VerletList(pd_vl h, long n) : h_(h), n_(n) {}
    VerletList(const VerletList&) = delete;
    VerletList& operator=(const VerletList&) = delete;
    VerletList(VerletList&& o) noexcept : h_(o.h_), n_(o.n_) { o.h_ = nullptr; }
    VerletList& operator=(VerletList&& o) noexcept {
        std::swap(h_, o.h_);
        std::swap(n_, o.n_);
        return *this;
    }
    ~VerletList() {
        if (h_) pd_verlet_destroy(h_);
    }
    pd_vl handle() const { return h_; }
    void set_size(long n) { n_ = n; }
    // CSR copy of the rows (getNNPart / get(i,j) of the reference's VerletList)
    void download(std::vector<int>& counts, std::vector<long>& offsets, std::vector<int>& idx) const {
        counts.assign(n_, 0);
        if (n_ == 0) return;
        check(pd_verlet_get(h_, counts.data(), nullptr, 0, nullptr));
        offsets.assign(n_ + 1, 0);
        for (long i = 0; i < n_; ++i) offsets[i + 1] = offsets[i] + counts[i];
        idx.assign(offsets[n_], 0);
        check(pd_verlet_get(h_, counts.data(), idx.data(), (long)idx.size(), nullptr));
    }
};

template <typename St> class vector_dist_gpu {
    static_assert(std::is_same<St, float>::value || std::is_same<St, double>::value, "St must be float or double");
    pd_vd h_ = nullptr;
    std::vector<prop_desc> props_;
    std::vector<St> pos_;                      // host mirror, AoS xyz
    std::vector<std::vector<unsigned char>> prp_;  // host mirrors, component-major [ncomp][mcap_]
    long mcap_ = 0;                            // particles the host mirrors hold room for
    long pending_ = 0;                         // particles added on the host, not yet on the device
    void* stream_ = nullptr;

    long size_all() const {
        long a = 0, b = 0;
        check(pd_size(h_, &a, &b));
        return b + pending_;
    }
    // room for n particles in the host mirrors (component columns moved to the new stride)
    void mirror(long n) {
        if (n <= mcap_) return;
        long nc = std::max<long>(n, 2 * mcap_);
        pos_.resize(3 * (size_t)nc);
        for (size_t p = 0; p < props_.size(); ++p) {
            const size_t es = (size_t)type_bytes(props_[p].type);
            std::vector<unsigned char> t((size_t)nc * props_[p].ncomp * es, 0);
            for (int c = 0; c < props_[p].ncomp && mcap_ > 0; ++c)
                std::copy(prp_[p].begin() + (size_t)c * mcap_ * es, prp_[p].begin() + (size_t)(c + 1) * mcap_ * es,
                          t.begin() + (size_t)c * nc * es);
            prp_[p].swap(t);
        }
        mcap_ = nc;
    }
    long device_all() const {
        long a = 0, b = 0;
        check(pd_size(h_, &a, &b));
        return b;
    }
    // the device vector takes the particles added on the host
    void flush_added() {
        if (pending_ == 0) return;
        long a = 0, b = 0;
        check(pd_size(h_, &a, &b));
        check(pd_resize(h_, a + pending_));
        pending_ = 0;
    }

  public:
    static constexpr int dims = 3;
    typedef St stype;

    vector_dist_gpu(long n, const std::array<double, 3>& lo, const std::array<double, 3>& hi,
                    const std::array<int, 3>& bc, const std::array<double, 3>& ghost,
                    const std::vector<prop_desc>& props = {}, void* stream = nullptr)
        : props_(props), prp_(props.size()), stream_(stream) {
        check(pd_create(3, std::is_same<St, double>::value ? PD_F64 : PD_F32, n, lo.data(), hi.data(), bc.data(),
                        ghost.data(), 0, &h_));
        for (auto& p : props_) {
            int id = -1;
            check(pd_add_prop(h_, p.type, p.ncomp, &id));
        }
        mirror(n);
    }
    vector_dist_gpu(const vector_dist_gpu&) = delete;
    vector_dist_gpu& operator=(const vector_dist_gpu&) = delete;
    ~vector_dist_gpu() {
        if (h_) pd_destroy(h_);
    }
    pd_vd handle() const { return h_; }

    long size_local() const {
        long a = 0, b = 0;
        check(pd_size(h_, &a, &b));
        return a + pending_;
    }
    long size_local_with_ghost() const { return size_all(); }

    // host mirror accessors (getPos(p)[k], getProp<prp>(p)[k])
    St* getPos(long p) { return pos_.data() + 3 * p; }
    template <typename T> T& getProp(int prp, long p, int comp = 0) {
        return reinterpret_cast<T*>(prp_[prp].data())[(long)comp * mcap_ + p];
    }
    // add() / getLastPos() / getLastProp -- vector_dist.hpp:923-984: a particle appended
    // on the host; the device vector takes it at the next hostToDevicePos/Prop
    void add() {
        mirror(size_local() + 1);
        ++pending_;
    }
    St* getLastPos() { return getPos(size_local() - 1); }
    template <typename T> T& getLastProp(int prp, int comp = 0) { return getProp<T>(prp, size_local() - 1, comp); }

    void hostToDevicePos() {
        flush_added();
        check(pd_h2d_pos(h_, pos_.data(), 0, size_local(), stream_));
    }
    void deviceToHostPos() {
        long n = device_all();
        mirror(n);
        if (n) check(pd_d2h_pos(h_, pos_.data(), 0, n, stream_));
    }
    void hostToDeviceProp(int prp) {
        flush_added();
        long n = size_local();
        // pack [ncomp][n] from the [ncomp][mcap_] mirror
        std::vector<unsigned char> tmp((size_t)n * props_[prp].ncomp * type_bytes(props_[prp].type));
        int es = type_bytes(props_[prp].type);
        for (int c = 0; c < props_[prp].ncomp; ++c)
            std::copy(prp_[prp].begin() + (size_t)c * mcap_ * es, prp_[prp].begin() + ((size_t)c * mcap_ + n) * es,
                      tmp.begin() + (size_t)c * n * es);
        check(pd_h2d_prop(h_, prp, tmp.data(), 0, n, stream_));
    }
    void deviceToHostProp(int prp) {
        long n = device_all();
        mirror(n);
        if (n == 0) return;
        // [ncomp][n] from the device, spread to the [ncomp][mcap_] mirror
        const int es = type_bytes(props_[prp].type);
        std::vector<unsigned char> tmp((size_t)n * props_[prp].ncomp * es);
        check(pd_d2h_prop(h_, prp, tmp.data(), 0, n, stream_));
        for (int c = 0; c < props_[prp].ncomp; ++c)
            std::copy(tmp.begin() + (size_t)c * n * es, tmp.begin() + (size_t)(c + 1) * n * es,
                      prp_[prp].begin() + (size_t)c * mcap_ * es);
    }

    // map(RUN_ON_DEVICE) -- vector_dist.hpp:2158
    void map(int opt = PD_RUN_ON_DEVICE) { check(pd_map(h_, opt, stream_)); }
    // ghost_get<prp...>(opt) -- vector_dist.hpp:2203
    void ghost_get(std::initializer_list<int> prps = {}, int opt = PD_RUN_ON_DEVICE) {
        unsigned long mask = 0;
        for (int p : prps) mask |= 1ul << p;
        if (prps.size() == 0) mask = ~0ul;
        check(pd_ghost_get(h_, mask, opt, stream_));
    }
    // Ighost_get<prp...>(opt) / ghost_wait() -- vector_dist.hpp:2241-2291
    void Ighost_get(std::initializer_list<int> prps = {}, int opt = PD_RUN_ON_DEVICE) {
        unsigned long mask = 0;
        for (int p : prps) mask |= 1ul << p;
        if (prps.size() == 0) mask = ~0ul;
        check(pd_ighost_get(h_, mask, opt, stream_));
    }
    void ghost_wait() { check(pd_ghost_wait(h_, stream_)); }
    // ghost_put<op_, prp...>() on one process -- vector_dist.hpp:2304 (op: PD_PUT_ADD / _MAX / _REPLACE)
    void ghost_put(std::initializer_list<int> prps = {}, int op = PD_PUT_ADD) {
        unsigned long mask = 0;
        for (int p : prps) mask |= 1ul << p;
        if (prps.size() == 0) mask = ~0ul;
        check(pd_ghost_put(h_, mask, op, stream_));
    }
    // getCellListSym(r_cut) -- vector_dist.hpp:1062
    CellList_gpu getCellListSym(St r_cut) { return getCellListGPU(r_cut, PD_CL_SYMMETRIC); }
    // getCellListGPU(r_cut, opt, NNIteratorBox, no_se3, ghostEnlargeFactor) -- vector_dist.hpp:1222
    CellList_gpu getCellListGPU(St r_cut, int opt = PD_CL_NON_SYMMETRIC, int nn_box = 1,
                                double enlarge = (double)1.013f) {
        pd_cl c = nullptr;
        check(pd_celllist_create(h_, (double)r_cut, opt, nn_box, enlarge, &c));
        return CellList_gpu(c);
    }
    // updateCellListGPU<prp...>(cl) -- vector_dist.hpp:1334
    void updateCellListGPU(CellList_gpu& cl, std::initializer_list<int> prps = {}) {
        unsigned long mask = 0;
        for (int p : prps) mask |= 1ul << p;
        check(pd_celllist_update(h_, cl.handle(), mask, stream_));
    }
    // restoreOrder<prp...>(cl) -- vector_dist.hpp:3042
    void restoreOrder(CellList_gpu& cl, std::initializer_list<int> prps = {}) {
        unsigned long mask = 0;
        for (int p : prps) mask |= 1ul << p;
        check(pd_restore_order(h_, cl.handle(), mask, stream_));
    }
    // getVerlet(r_cut) / updateVerlet(vl) -- vector_dist.hpp:1514-1620
    VerletList getVerlet(St r_cut) {
        pd_vl v = nullptr;
        check(pd_verlet_create(h_, (double)r_cut, &v));
        VerletList vl(v, size_local());
        check(pd_verlet_update(h_, v, stream_));
        return vl;
    }
    // getVerletSym(r_cut) -- vector_dist.hpp:1412
    VerletList getVerletSym(St r_cut) {
        pd_vl v = nullptr;
        check(pd_verlet_create_sym(h_, (double)r_cut, &v));
        VerletList vl(v, size_local());
        check(pd_verlet_update(h_, v, stream_));
        return vl;
    }
    // save(filename) / load(filename) -- vector_dist.hpp:2459-2476 (own checksummed binary format)
    void save(const std::string& path) const { check(pd_save(h_, path.c_str())); }
    void load(const std::string& path) { check(pd_load(h_, path.c_str())); }
    // write(out, meta_info, opt) / write_frame(out, iteration, meta_info, opt) -- vector_dist.hpp:2498-2721
    void write(const std::string& out, const std::string& meta = "", int opt = PD_VTK_WRITER) const {
        check(pd_write(h_, out.c_str(), meta.c_str(), opt));
    }
    void write_frame(const std::string& out, long iteration, const std::string& meta = "",
                     int opt = PD_VTK_WRITER) const {
        check(pd_write_frame(h_, out.c_str(), iteration, meta.c_str(), opt));
    }
    // remove_marked<prp>(vd) -- vector_dist_cuda_funcs.cuh:333
    void remove_marked(int prp) { check(pd_remove_marked(h_, prp, stream_)); }
    // get_indexes_by_type<prp, functor>(vd, ids, end) -- vector_dist_cuda_funcs.cuh:449;
    // the functor's check as a comparison cmp (PD_CMP_*) with value
    std::vector<unsigned int> get_indexes_by_type(int prp, int cmp, long long value, long end = -1) {
        std::vector<unsigned int> ids((size_t)(size_all() > 0 ? size_all() : 1));
        long n = 0;
        check(pd_get_indexes_by_type(h_, prp, cmp, value, end, ids.data(), (long)ids.size(), &n, stream_));
        ids.resize((size_t)n);
        return ids;
    }
    // the same into caller-owned device memory of `cap` entries (as the reference's
    // vector_gpu keeps them on the device); returns the number of indexes
    long get_indexes_by_type(int prp, int cmp, long long value, unsigned int* ids_dev, long cap, long end = -1) {
        long n = 0;
        check(pd_get_indexes_by_type(h_, prp, cmp, value, end, ids_dev, cap, &n, stream_));
        return n;
    }
    void updateVerlet(VerletList& vl) {
        check(pd_verlet_update(h_, vl.handle(), stream_));
        vl.set_size(size_local());
    }
    // getDomainIteratorGPU(n_thr) -- vector_dist.hpp:1958
    pd_launch_t getDomainIteratorGPU(int n_thr = 1024) const {
        pd_launch_t it;
        check(pd_domain_iterator(h_, n_thr, 0, &it));
        return it;
    }
    pd_launch_t getDomainAndGhostIteratorGPU(int n_thr = 1024) const {
        pd_launch_t it;
        check(pd_domain_iterator(h_, n_thr, 1, &it));
        return it;
    }
    // toKernel() -- vector_dist.hpp:2961
    pd_view_t toKernel() const {
        pd_view_t v;
        check(pd_view(h_, &v));
        return v;
    }
    // reduce_local<prp,_add_/_max_> -- vector_dist_cuda_funcs.cuh:247
    double reduce_local(int prp, int comp, int op) {
        double out = 0;
        check(pd_reduce(h_, prp, comp, op, stream_, &out));
        return out;
    }
};

// velocity-Verlet LJ driver
class md_lj {
    pd_md h_ = nullptr;

  public:
    template <typename St>
    md_lj(vector_dist_gpu<St>& vd, pd_lj_params_t lj, pd_md_params_t mp) {
        check(pd_md_create(vd.handle(), &lj, &mp, &h_));
    }
    md_lj(const md_lj&) = delete;
    md_lj& operator=(const md_lj&) = delete;
    ~md_lj() {
        if (h_) pd_md_destroy(h_);
    }
    // run `steps` steps; returns [steps][4] = KE, PE, virial, rebuilt
    std::vector<double> run(int steps, void* stream = nullptr) {
        std::vector<double> E(4 * (size_t)(steps > 0 ? steps : 1));
        check(pd_md_run(h_, steps, stream, E.data()));
        E.resize(4 * (size_t)steps);
        return E;
    }
};

}  // namespace pd
