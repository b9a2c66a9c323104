// C++ host program over include/pd/vector_dist_gpu.hpp: the reference-style loop
// (map, ghost_get, getVerlet, LJ forces) followed by the velocity-Verlet driver.
// Reads "n L" and n lines of "x y z vx vy vz" from stdin; prints
//   pairs <sum of Verlet row lengths>
//   E <KE> <PE> <virial> <rebuilt>   (one line per step)
#include <cstdio>
#include <vector>

#include "pd/vector_dist_gpu.hpp"

int main(int argc, char** argv) {
    int steps = argc > 1 ? atoi(argv[1]) : 10;
    long n;
    double L;
    if (scanf("%ld %lf", &n, &L) != 2) return 2;
    // an empty vector filled with add() / getLastPos() / getLastProp, as the reference's examples do
    pd::vector_dist_gpu<double> vd(0, {0, 0, 0}, {L, L, L}, {PD_PERIODIC, PD_PERIODIC, PD_PERIODIC},
                                   {2.8, 2.8, 2.8}, {{PD_F64, 3}, {PD_F64, 3}});
    for (long i = 0; i < n; ++i) {
        vd.add();
        double* x = vd.getLastPos();
        double v[3];
        if (scanf("%lf %lf %lf %lf %lf %lf", &x[0], &x[1], &x[2], &v[0], &v[1], &v[2]) != 6) return 2;
        for (int d = 0; d < 3; ++d) vd.getLastProp<double>(0, d) = v[d];
    }
    if (vd.size_local() != n) return 3;
    vd.hostToDevicePos();
    vd.hostToDeviceProp(0);
    vd.map();
    vd.ghost_get();
    auto vl = vd.getVerlet(2.8);
    std::vector<int> counts, idx;
    std::vector<long> off;
    vl.download(counts, off, idx);
    printf("pairs %ld\n", off.empty() ? 0L : off.back());
    vd.map();  // drop the ghost before handing the vector to the integrator
    pd::md_lj md(vd, pd_lj_params_t{1.0, 1.0, 2.5}, pd_md_params_t{0.005, 1.0, 0.3, 0, 1, 0, PD_PREC_FP64});
    std::vector<double> E = md.run(steps);
    for (int s = 0; s < steps; ++s) printf("E %.17g %.17g %.17g %.0f\n", E[4 * s], E[4 * s + 1], E[4 * s + 2], E[4 * s + 3]);
    return 0;
}
