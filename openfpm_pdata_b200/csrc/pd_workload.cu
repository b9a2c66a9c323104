// pd_workload.cu -- host generator of the clustered LJ layout (64 Gaussian
// clusters with a minimum-distance rejection), too slow in Python at 4M
// particles.  Host code only; no device work.
//
// Rules: cluster centres uniform in [0, L)^3; particle i belongs to cluster
// i / ceil(n / n_clusters); candidate = centre + N(0, sigma_c) per axis, wrapped
// into the periodic box; a candidate closer than min_dist (minimum image) to an
// accepted particle is redrawn, at most max_tries times, after which the
// cluster's centre is redrawn uniformly (the core density of 64k particles in
// a sigma_c = 8 Gaussian exceeds what a 0.8 minimum distance allows, so cores
// saturate and clusters spread).  Acceptance is checked on a grid of cells of
// side >= min_dist (27 cells).  std::mt19937_64, seeded.
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

#include "pd_internal.cuh"

extern "C" int pd_gen_clustered(long n, double L, int n_clusters, double sigma_c, double min_dist, unsigned long seed,
                                int max_tries, double* x_out, long* centre_redraws) {
    if (n < 1 || !(L > 0) || n_clusters < 1 || !(sigma_c > 0) || !(min_dist > 0) || max_tries < 1 || !x_out)
        return PD_EINVAL;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(0.0, L);
    std::normal_distribution<double> N(0.0, sigma_c);
    std::vector<double> cx(3 * (size_t)n_clusters);
    for (auto& c : cx) c = U(rng);
    long nc = (long)std::floor(L / min_dist);
    if (nc < 3) nc = 3;
    if (nc > 1024) nc = 1024;
    const double side = L / (double)nc;
    std::vector<int> head((size_t)nc * nc * nc, -1);
    std::vector<int> next((size_t)n, -1);
    const long per = (n + n_clusters - 1) / n_clusters;
    const double md2 = min_dist * min_dist;
    long redraws = 0;
    auto wrap = [L](double v) {
        v = std::fmod(v, L);
        if (v < 0) v += L;
        if (v >= L) v = 0.0;
        return v;
    };
    auto cell = [&](double v) {
        long c = (long)std::floor(v / side);
        return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
    };
    for (long i = 0; i < n; ++i) {
        const int k = (int)std::min((long)n_clusters - 1, i / per);
        int tries = 0;
        double p[3];
        long c[3];
        for (;;) {
            for (int d = 0; d < 3; ++d) {
                p[d] = wrap(cx[3 * k + d] + N(rng));
                c[d] = cell(p[d]);
            }
            bool ok = true;
            for (int dz = -1; dz <= 1 && ok; ++dz)
                for (int dy = -1; dy <= 1 && ok; ++dy)
                    for (int dx = -1; dx <= 1 && ok; ++dx) {
                        const long a = (c[0] + dx + nc) % nc, b = (c[1] + dy + nc) % nc, e = (c[2] + dz + nc) % nc;
                        for (int q = head[(size_t)a + nc * (b + nc * e)]; q >= 0; q = next[q]) {
                            double r2 = 0;
                            for (int d = 0; d < 3; ++d) {
                                double t = p[d] - x_out[3 * (size_t)q + d];
                                t -= L * std::round(t / L);
                                r2 += t * t;
                            }
                            if (r2 < md2) {
                                ok = false;
                                break;
                            }
                        }
                    }
            if (ok) break;
            if (++tries >= max_tries) {
                for (int d = 0; d < 3; ++d) cx[3 * k + d] = U(rng);
                ++redraws;
                tries = 0;
            }
        }
        for (int d = 0; d < 3; ++d) x_out[3 * (size_t)i + d] = p[d];
        const size_t h = (size_t)c[0] + nc * (c[1] + nc * c[2]);
        next[i] = head[h];
        head[h] = (int)i;
    }
    if (centre_redraws) *centre_redraws = redraws;
    return PD_OK;
}
