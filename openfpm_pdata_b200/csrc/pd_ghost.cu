// pd_ghost.cu -- ghost_get on one GPU: periodic images of the real particles.
//
// The reference (one process) runs num_shift_ghost_each_part -> scan ->
// shift_ghost_each_part over the local ghost boxes sorted by shift id
// (vector_dist_comm_util_funcs.cuh:247-304, vector_dist_cuda_funcs.cuh:157-233),
// and with SKIP_LABELLING replays the stored (particle, shift) list
// (process_ghost_particles_local, :133-155).  Here the same three passes run
// with the box list resident in device memory, the scan total stays on the
// device (the control block) so the image build can also run without a host
// round trip, and image records are kept for the replay.
#include "pd_device.cuh"
#include "pd_internal.cuh"
#include "pd_ghost_dev.cuh"

namespace pd {

struct PropCopy {
    char* d[16];
    int esize[16];
    int ncomp[16];
    int n;
    long cap;
};

__device__ __forceinline__ void copy_props(const PropCopy& pc, long from, long to) {
    for (int p = 0; p < pc.n; ++p) {
        char* base = pc.d[p];
        if (pc.esize[p] == 8) {
            for (int c = 0; c < pc.ncomp[p]; ++c) {
                long long* a = reinterpret_cast<long long*>(base) + (long)c * pc.cap;
                a[to] = a[from];
            }
        } else {
            for (int c = 0; c < pc.ncomp[p]; ++c) {
                int* a = reinterpret_cast<int*>(base) + (long)c * pc.cap;
                a[to] = a[from];
            }
        }
    }
}

// num_shift_ghost_each_part
template <class T>
__global__ void k_ghost_count(const typename V4<T>::type* __restrict__ pos, long n, const BoxSet<T>* __restrict__ Bp,
                              unsigned int* __restrict__ cnt) {
    __shared__ BoxSet<T> B;
    for (int i = threadIdx.x; i < (int)(sizeof(BoxSet<T>) / 4); i += blockDim.x)
        reinterpret_cast<int*>(&B)[i] = reinterpret_cast<const int*>(Bp)[i];
    __syncthreads();
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
        typename V4<T>::type r = ld4(pos, p);
        unsigned int c = 0;
        int old = -1;
        const int nb = in_core(B, r.x, r.y, r.z) ? 0 : B.nb;
        for (int i = 0; i < nb; ++i) {
            int s = B.sv[i];
            if (inside_np(B, i, r.x, r.y, r.z) && s != old) {
                old = s;
                c++;
            }
        }
        cnt[p] = c;
    }
}

// shift_ghost_each_part: image j of particle p goes to slot n + start[p] + j
template <class T>
__global__ void k_ghost_write(typename V4<T>::type* __restrict__ pos, int* __restrict__ gid, long n,
                              const BoxSet<T>* __restrict__ Bp, const T* __restrict__ shifts,
                              const unsigned int* __restrict__ start, int* __restrict__ src,
                              unsigned char* __restrict__ shf, long img_cap, long cap, PropCopy pc,
                              unsigned int* __restrict__ err) {
    __shared__ BoxSet<T> B;
    for (int i = threadIdx.x; i < (int)(sizeof(BoxSet<T>) / 4); i += blockDim.x)
        reinterpret_cast<int*>(&B)[i] = reinterpret_cast<const int*>(Bp)[i];
    __syncthreads();
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
        typename V4<T>::type r = ld4(pos, p);
        long m = start[p];
        int old = -1;
        const int nb = in_core(B, r.x, r.y, r.z) ? 0 : B.nb;
        for (int i = 0; i < nb; ++i) {
            int s = B.sv[i];
            if (inside_np(B, i, r.x, r.y, r.z) && s != old) {
                old = s;
                if (m < img_cap && n + m < cap) {
                    typename V4<T>::type q;
                    q.x = r.x - shifts[3 * s];
                    q.y = r.y - shifts[3 * s + 1];
                    q.z = r.z - shifts[3 * s + 2];
                    q.w = r.w;
                    st4(pos, n + m, q);
                    gid[n + m] = gid[p];
                    src[m] = (int)p;
                    shf[m] = (unsigned char)s;
                    copy_props(pc, p, n + m);
                } else {
                    atomicOr(err, ERR_IMG_OVERFLOW);
                }
                m++;
            }
        }
    }
}

// process_ghost_particles_local: replay the stored image list
template <class T>
__global__ void k_ghost_replay(typename V4<T>::type* __restrict__ pos, long n, const int* __restrict__ src,
                               const unsigned char* __restrict__ shf, const T* __restrict__ shifts,
                               const unsigned int* __restrict__ n_img_dev, long n_img_bound, int with_pos,
                               PropCopy pc) {
    long m_n = n_img_dev ? (long)*n_img_dev : n_img_bound;
    if (m_n > n_img_bound) m_n = n_img_bound;
    for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < m_n; m += (long)gridDim.x * blockDim.x) {
        int p = src[m];
        if (with_pos) {
            int s = shf[m];
            typename V4<T>::type r = ld4(pos, p);
            r.x -= shifts[3 * s];
            r.y -= shifts[3 * s + 1];
            r.z -= shifts[3 * s + 2];
            st4(pos, n + m, r);
        }
        if (pc.n) copy_props(pc, p, n + m);
    }
}

// ghost_put<op, prp...> on one process (vector_dist_comm.hpp:2086-2182, the local
// part merge_prp_v): every image's value is merged onto its source in image
// order -- the images of a source are consecutive (generation order), so one
// thread per source applies them in that order and the result is deterministic.
template <class E>
__global__ void k_ghost_put(E* __restrict__ a, long cap, int ncomp, long n, const unsigned int* __restrict__ start,
                            const unsigned int* __restrict__ cnt, int op) {
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
        const unsigned int m = cnt[p];
        if (m == 0) continue;
        const long base = n + (long)start[p];
        for (int c = 0; c < ncomp; ++c) {
            E* col = a + (long)c * cap;
            E acc = col[p];
            for (unsigned int j = 0; j < m; ++j) {
                const E v = col[base + j];
                acc = op == PD_PUT_ADD ? acc + v : (op == PD_PUT_MAX ? (v > acc ? v : acc) : v);
            }
            col[p] = acc;
        }
    }
}

static PropCopy make_copy(pd_vd h, unsigned long mask) {
    PropCopy pc;
    memset(&pc, 0, sizeof(pc));
    pc.cap = h->cap;
    for (size_t p = 0; p < h->props.size(); ++p) {
        if (!(mask & (1ul << p))) continue;
        pc.d[pc.n] = h->props[p].d;
        pc.esize[pc.n] = h->props[p].esize;
        pc.ncomp[pc.n] = h->props[p].ncomp;
        pc.n++;
    }
    return pc;
}

// Local periodic ghost boxes of one sub-domain equal to the domain, sorted by
// shift id: the replica of the domain shifted by -L*c (applyBC,
// ie_loc_ghost.hpp:145-200) enlarged by the ghost and intersected with the
// domain (create_loc_ghost_ibox, :102-143); shift vectors -L*c indexed by
// c.lin() (shift_vect_converter.hpp:36-66).
template <class T> static int domain_boxes(pd_vd h, BoxSet<T>& B, T* shifts) {
    T lo[3], hi[3], g[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = (T)h->lo[d];
        hi[d] = (T)h->hi[d];
        g[d] = (T)h->g[d];
    }
    B.nb = 0;
    B.core = 0;
    for (int l = 0; l < 27; ++l) {
        int c[3] = {l % 3 - 1, (l / 3) % 3 - 1, l / 9 - 1};
        for (int d = 0; d < 3; ++d)
            shifts[3 * l + d] = c[d] == 1 ? -(hi[d] - lo[d]) : (c[d] == -1 ? (hi[d] - lo[d]) : T(0));
        if (c[0] == 0 && c[1] == 0 && c[2] == 0) continue;
        bool ok = true;
        for (int d = 0; d < 3; ++d)
            if (c[d] != 0 && h->bc[d] != PD_PERIODIC) ok = false;
        if (!ok) continue;
        bool empty = false;
        T bl[3], bu[3];
        for (int d = 0; d < 3; ++d) {
            T sh = c[d] == 1 ? (-hi[d] + lo[d]) : (c[d] == -1 ? (hi[d] - lo[d]) : T(0));
            T el = (lo[d] + sh) + (-g[d]), eu = (hi[d] + sh) + g[d];
            bl[d] = lo[d] > el ? lo[d] : el;
            bu[d] = hi[d] < eu ? hi[d] : eu;
            if (bl[d] >= bu[d]) empty = true;
        }
        if (empty) continue;
        for (int d = 0; d < 3; ++d) {
            B.lo[B.nb][d] = bl[d];
            B.hi[B.nb][d] = bu[d];
        }
        B.sv[B.nb] = l;
        B.nb++;
    }
    return B.nb;
}

// The core of a box set inside the domain: on each axis, between the highest box
// upper edge at or below the middle and the lowest box lower edge at or above it
// (boxes across the middle leave that axis open).  Kept only if it is not empty and
// every box misses it on some axis, so that no point of it lies in a box.
template <class T> static void box_core(pd_vd h, BoxSet<T>& B) {
    B.core = 0;
    if (B.nb <= 0) return;
    for (int d = 0; d < 3; ++d) {
        const T lo = (T)h->lo[d], hi = (T)h->hi[d], mid = lo + (hi - lo) / T(2);
        T cl = lo, ch = hi;
        for (int i = 0; i < B.nb; ++i) {
            if (B.hi[i][d] <= mid && B.hi[i][d] > cl) cl = B.hi[i][d];
            if (B.lo[i][d] >= mid && B.lo[i][d] < ch) ch = B.lo[i][d];
        }
        if (!(cl < ch)) return;
        B.clo[d] = cl;
        B.chi[d] = ch;
    }
    for (int i = 0; i < B.nb; ++i) {
        bool misses = false;
        for (int d = 0; d < 3; ++d)
            if (B.hi[i][d] <= B.clo[d] || B.lo[i][d] >= B.chi[d]) misses = true;
        if (!misses) return;
    }
    B.core = 1;
}

template <class T> static int upload_boxes_t(pd_vd h, const BoxSet<T>& B_in, const T* shifts, int n_shifts,
                                             cudaStream_t st) {
    BoxSet<T> B = B_in;
    box_core(h, B);
    PD_TRY(h->boxes.ensure(sizeof(BoxSet<T>)));
    PD_TRY(h->shifts.ensure(sizeof(T) * 3 * (n_shifts > 27 ? n_shifts : 27)));
    PD_CUDA(cudaMemcpyAsync(h->boxes.p, &B, sizeof(BoxSet<T>), cudaMemcpyHostToDevice, st));
    PD_CUDA(cudaMemcpyAsync(h->shifts.p, shifts, sizeof(T) * 3 * n_shifts, cudaMemcpyHostToDevice, st));
    PD_CUDA(cudaStreamSynchronize(st));  // host staging buffers are stack locals
    h->nbox = B.nb;
    return PD_OK;
}

int ghost_boxes_upload(pd_vd h, cudaStream_t st) {
    if (h->dtype == PD_F64) {
        BoxSet<double> B;
        double sh[81];
        domain_boxes(h, B, sh);
        return upload_boxes_t(h, B, sh, 27, st);
    } else {
        BoxSet<float> B;
        float sh[81];
        domain_boxes(h, B, sh);
        return upload_boxes_t(h, B, sh, 27, st);
    }
}

// domain ghost boxes and shift vectors of an FP64 vector into caller-owned host
// memory (no copy); the caller uploads them to h->boxes / h->shifts
int ghost_boxes_host(pd_vd h, BoxSet<double>* B, double* shifts27) {
    if (h->dtype != PD_F64) return PD_EINVAL;
    domain_boxes(h, *B, shifts27);
    return PD_OK;
}

// count -> scan (total to the control block) -> write.  With sync_count the
// total is read back and the capacity grown (the API path, like the reference's
// D->H copy of the scan tail); without it `img_cap` bounds the write and an
// overflow sets ERR_IMG_OVERFLOW (the captured integrator path).
int ghost_generate(pd_vd h, long img_cap, bool sync_count, cudaStream_t st) {
    long n = h->n_real;
    PD_TRY(h->img_cnt.ensure(sizeof(unsigned int) * (n + 1)));
    PD_TRY(h->img_start.ensure(sizeof(unsigned int) * (n + 1)));
    unsigned g = grid_for(n, 256);
    if (n > 0) {
        if (h->dtype == PD_F64)
            pd::launch(k_ghost_count<double>, g, 256, 0, st, (const double4*)h->pos, n, h->boxes.as<BoxSet<double>>(),
                                                     h->img_cnt.as<unsigned int>());
        else
            pd::launch(k_ghost_count<float>, g, 256, 0, st, (const float4*)h->pos, n, h->boxes.as<BoxSet<float>>(),
                                                    h->img_cnt.as<unsigned int>());
        PD_LAUNCH_CHECK();
    }
    PD_TRY(scan_u32(h->img_cnt.as<unsigned int>(), h->img_start.as<unsigned int>(), n, &h->ctrl->n_img,
                    h->scan_scratch, st));
    long m_cap = img_cap;
    if (sync_count) {
        PD_TRY(read_ctrl(h, st));
        long m = h->ctrl_h->n_img;
        PD_TRY(ensure_capacity(h, n + m + 1, st));
        m_cap = m;
    }
    if (m_cap < 1) m_cap = 1;
    PD_TRY(h->img_src.ensure(sizeof(int) * m_cap));
    PD_TRY(h->img_shift.ensure(m_cap));
    if (n > 0) {
        PropCopy pc = make_copy(h, ~0ul);
        if (h->dtype == PD_F64)
            pd::launch(k_ghost_write<double>, g, 256, 0, st, (double4*)h->pos, h->gid, n, h->boxes.as<BoxSet<double>>(),
                                                     h->shifts.as<double>(), h->img_start.as<unsigned int>(),
                                                     h->img_src.as<int>(), h->img_shift.as<unsigned char>(), m_cap,
                                                     h->cap, pc, &h->ctrl->err);
        else
            pd::launch(k_ghost_write<float>, g, 256, 0, st, (float4*)h->pos, h->gid, n, h->boxes.as<BoxSet<float>>(),
                                                    h->shifts.as<float>(), h->img_start.as<unsigned int>(),
                                                    h->img_src.as<int>(), h->img_shift.as<unsigned char>(), m_cap,
                                                    h->cap, pc, &h->ctrl->err);
        PD_LAUNCH_CHECK();
    }
    if (sync_count) {
        h->n_img = h->ctrl_h->n_img;
        h->n_total = n + h->n_img;
        h->img_valid = true;
        h->img_gen_order = true;
    }
    return PD_OK;
}

int ghost_replay(pd_vd h, unsigned long prop_mask, bool with_pos, const unsigned int* n_img_dev, long n_img_bound,
                 cudaStream_t st) {
    if (n_img_bound <= 0) return PD_OK;
    PropCopy pc = make_copy(h, prop_mask);
    unsigned g = grid_for(n_img_bound, 256);
    if (h->dtype == PD_F64)
        pd::launch(k_ghost_replay<double>, g, 256, 0, st, (double4*)h->pos, h->n_real, h->img_src.as<int>(),
                                                  h->img_shift.as<unsigned char>(), h->shifts.as<double>(),
                                                  n_img_dev, n_img_bound, with_pos ? 1 : 0, pc);
    else
        pd::launch(k_ghost_replay<float>, g, 256, 0, st, (float4*)h->pos, h->n_real, h->img_src.as<int>(),
                                                 h->img_shift.as<unsigned char>(), h->shifts.as<float>(), n_img_dev,
                                                 n_img_bound, with_pos ? 1 : 0, pc);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

template <class T> static int user_boxes(pd_vd h, const double* boxes, const int* sv, int nb, BoxSet<T>& B) {
    if (nb < 0 || nb > MAXBOX) {
        set_error("at most %d ghost boxes", MAXBOX);
        return PD_EINVAL;
    }
    memset(&B, 0, sizeof(B));
    B.nb = nb;
    for (int i = 0; i < nb; ++i) {
        for (int d = 0; d < 3; ++d) {
            B.lo[i][d] = (T)boxes[6 * i + d];
            B.hi[i][d] = (T)boxes[6 * i + 3 + d];
        }
        if (sv[i] < 0 || sv[i] > 255) {
            set_error("shift id out of range");
            return PD_EINVAL;
        }
        B.sv[i] = sv[i];
    }
    return PD_OK;
}

}  // namespace pd

using namespace pd;

extern "C" {

int pd_ghost_get(pd_vd h, unsigned long prop_mask, int opt, void* stream) {
    if (!h) return PD_EINVAL;
    if (h->ghost_pending) {
        set_error("ghost_get: an Ighost_get is waiting for its ghost_wait");
        return PD_ESTATE;
    }
    cudaStream_t st = S(stream);
    if ((opt & PD_SKIP_LABELLING) && h->img_valid) {
        // ghost_get_ with SKIP_LABELLING: positions unless NO_POSITION, properties in the mask
        PD_TRY(ghost_replay(h, prop_mask, !(opt & PD_NO_POSITION), nullptr, h->n_img, st));
        return PD_OK;
    }
    h->n_total = h->n_real;
    PD_TRY(ghost_boxes_upload(h, st));
    PD_TRY(ghost_generate(h, 0, true, st));
    PD_TRY(read_ctrl(h, st));
    if (h->ctrl_h->err & ERR_IMG_OVERFLOW) {
        set_error("ghost_get: image overflow");
        return PD_EOVERFLOW;
    }
    h->epoch++;
    return PD_OK;
}

int pd_ighost_get(pd_vd h, unsigned long prop_mask, int opt, void* stream) {
    if (!h) return PD_EINVAL;
    if (h->ghost_pending) {
        set_error("Ighost_get: the previous Ighost_get was not waited for");
        return PD_ESTATE;
    }
    cudaStream_t st = S(stream);
    h->pend_mask = prop_mask;
    h->pend_opt = opt;
    if ((opt & PD_SKIP_LABELLING) && h->img_valid) {
        PD_TRY(ghost_replay(h, prop_mask, !(opt & PD_NO_POSITION), nullptr, h->n_img, st));
        h->ghost_pending = true;
        h->pend_replay = true;
        return PD_OK;
    }
    // images written without a host read of their count: room for the previous count
    // with a margin (growing the storage, if needed, synchronises once here); an
    // overflow is detected by ghost_wait, which then redoes the call synchronously
    h->n_total = h->n_real;
    h->img_valid = false;
    const long want = h->n_img + h->n_img / 4 + 1024;
    PD_TRY(ensure_capacity(h, h->n_real + want + 1, st));
    if (h->nbox == 0) PD_TRY(ghost_boxes_upload(h, st));
    PD_TRY(ghost_generate(h, h->cap - h->n_real - 1, false, st));
    h->ghost_pending = true;
    h->pend_replay = false;
    return PD_OK;
}

int pd_ghost_wait(pd_vd h, void* stream) {
    if (!h) return PD_EINVAL;
    if (!h->ghost_pending) return PD_OK;
    cudaStream_t st = S(stream);
    h->ghost_pending = false;
    if (h->pend_replay) return cudaStreamSynchronize(st) == cudaSuccess ? PD_OK : PD_ECUDA;
    PD_TRY(read_ctrl(h, st));
    if (h->ctrl_h->err & ERR_IMG_OVERFLOW) {
        h->ctrl_h->err &= ~ERR_IMG_OVERFLOW;
        PD_CUDA(cudaMemcpyAsync(&h->ctrl->err, &h->ctrl_h->err, sizeof(unsigned int), cudaMemcpyHostToDevice, st));
        return pd_ghost_get(h, h->pend_mask, h->pend_opt & ~PD_SKIP_LABELLING, stream);
    }
    h->n_img = h->ctrl_h->n_img;
    h->n_total = h->n_real + h->n_img;
    h->img_valid = true;
    h->img_gen_order = true;
    h->epoch++;
    return PD_OK;
}

int pd_ghost_put(pd_vd h, unsigned long prop_mask, int op, void* stream) {
    if (!h || (op != PD_PUT_ADD && op != PD_PUT_MAX && op != PD_PUT_REPLACE)) return PD_EINVAL;
    if (!h->img_valid || !h->img_gen_order) {
        set_error("ghost_put: no ghost_get images in generation order (call ghost_get first)");
        return PD_ESTATE;
    }
    cudaStream_t st = S(stream);
    const long n = h->n_real;
    if (n == 0 || h->n_img == 0) return PD_OK;
    const unsigned g = grid_for(n, 256);
    const unsigned int* start = h->img_start.as<unsigned int>();
    const unsigned int* cnt = h->img_cnt.as<unsigned int>();
    for (size_t p = 0; p < h->props.size(); ++p) {
        if (!(prop_mask & (1ul << p))) continue;
        Prop& P = h->props[p];
        switch (P.type) {
            case PD_F64: pd::launch(k_ghost_put<double>, g, 256, 0, st, (double*)P.d, h->cap, P.ncomp, n, start, cnt, op); break;
            case PD_F32: pd::launch(k_ghost_put<float>, g, 256, 0, st, (float*)P.d, h->cap, P.ncomp, n, start, cnt, op); break;
            case PD_I32: pd::launch(k_ghost_put<int>, g, 256, 0, st, (int*)P.d, h->cap, P.ncomp, n, start, cnt, op); break;
            case PD_U32: pd::launch(k_ghost_put<unsigned int>, g, 256, 0, st, (unsigned int*)P.d, h->cap, P.ncomp, n, start, cnt, op); break;
            case PD_I64: pd::launch(k_ghost_put<long long>, g, 256, 0, st, (long long*)P.d, h->cap, P.ncomp, n, start, cnt, op); break;
        }
        PD_LAUNCH_CHECK();
    }
    return PD_OK;
}

int pd_ghost_records(pd_vd h, int* src, int* shift_id, long cap, long* n_img) {
    if (!h || !n_img) return PD_EINVAL;
    *n_img = h->img_valid ? h->n_img : 0;
    long m = *n_img < cap ? *n_img : cap;
    if (m > 0) {
        if (src) PD_CUDA(cudaMemcpy(src, h->img_src.p, sizeof(int) * m, cudaMemcpyDeviceToHost));
        if (shift_id) {
            std::vector<unsigned char> t(m);
            PD_CUDA(cudaMemcpy(t.data(), h->img_shift.p, m, cudaMemcpyDeviceToHost));
            for (long i = 0; i < m; ++i) shift_id[i] = t[i];
        }
    }
    return PD_OK;
}

int pd_ghost_count_boxes(pd_vd h, const double* boxes_host, const int* sv_host, int nb, int* counts_host,
                         void* stream) {
    if (!h || !boxes_host || !sv_host || !counts_host) return PD_EINVAL;
    cudaStream_t st = S(stream);
    long n = h->n_real;
    PD_TRY(h->img_cnt.ensure(sizeof(unsigned int) * (n + 1)));
    unsigned g = grid_for(n, 256);
    if (h->dtype == PD_F64) {
        BoxSet<double> B;
        PD_TRY(user_boxes(h, boxes_host, sv_host, nb, B));
        double sh[3] = {0, 0, 0};
        PD_TRY(upload_boxes_t(h, B, sh, 1, st));
        if (n) pd::launch(k_ghost_count<double>, g, 256, 0, st, (const double4*)h->pos, n, h->boxes.as<BoxSet<double>>(),
                                                        h->img_cnt.as<unsigned int>());
    } else {
        BoxSet<float> B;
        PD_TRY(user_boxes(h, boxes_host, sv_host, nb, B));
        float sh[3] = {0, 0, 0};
        PD_TRY(upload_boxes_t(h, B, sh, 1, st));
        if (n) pd::launch(k_ghost_count<float>, g, 256, 0, st, (const float4*)h->pos, n, h->boxes.as<BoxSet<float>>(),
                                                       h->img_cnt.as<unsigned int>());
    }
    PD_LAUNCH_CHECK();
    if (n) PD_CUDA(cudaMemcpyAsync(counts_host, h->img_cnt.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    h->img_valid = false;  // the domain boxes were replaced
    h->nbox = 0;
    return PD_OK;
}

int pd_ghost_get_boxes(pd_vd h, const double* boxes_host, const int* sv_host, int nb, const double* shifts_host,
                       int n_shifts, void* stream) {
    if (!h || !boxes_host || !sv_host || !shifts_host || n_shifts < 1 || n_shifts > 256) return PD_EINVAL;
    for (int i = 0; i < nb; ++i)
        if (sv_host[i] >= n_shifts) {
            set_error("shift id %d has no shift vector", sv_host[i]);
            return PD_EINVAL;
        }
    cudaStream_t st = S(stream);
    h->n_total = h->n_real;
    if (h->dtype == PD_F64) {
        BoxSet<double> B;
        PD_TRY(user_boxes(h, boxes_host, sv_host, nb, B));
        PD_TRY(upload_boxes_t(h, B, shifts_host, n_shifts, st));
    } else {
        BoxSet<float> B;
        PD_TRY(user_boxes(h, boxes_host, sv_host, nb, B));
        std::vector<float> sh(3 * n_shifts);
        for (int i = 0; i < 3 * n_shifts; ++i) sh[i] = (float)shifts_host[i];
        PD_TRY(upload_boxes_t(h, B, sh.data(), n_shifts, st));
    }
    PD_TRY(ghost_generate(h, 0, true, st));
    PD_TRY(read_ctrl(h, st));
    h->nbox = 0;  // next domain ghost_get re-uploads the domain boxes
    h->epoch++;
    return (h->ctrl_h->err & ERR_IMG_OVERFLOW) ? PD_EOVERFLOW : PD_OK;
}

}  // extern "C"
