// gamera_gpu_x: a C++ host for the B200 GAMERA step that drives the C ABI (include/gamgpu.h) the way the
// reference's gamera.x drives stepGamera (src/drivers/gamerax.F90: InitModel, then AdvanceModel until
// tFin with console output at a step cadence). It builds one of the built-in problems from corner
// coordinates generated here, runs it on the current CUDA device and reports zone-updates/s.
//
//   gamera_gpu_x [--problem bw|ot|lfmbw] [--n N] [--steps K] [--prec fp64|fp32flux] [--ts-out M]
//                [--dump FILE]
//
// --dump writes State%Gas (Fortran layout, ghosts included, doubles) after the K stepped steps; the K
// device-timed steps that follow only measure throughput.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gamgpu.h"

namespace {

const double PI = 3.14159265358979323846264338327950288;

struct Opts {
    std::string problem = "bw";
    int n = 64, steps = 20, tsOut = 10;
    int prec = GAM_FP64;
    std::string dump;
};

Opts parse(int argc, char** argv) {
    Opts o;
    for (int a = 1; a < argc; ++a) {
        std::string s = argv[a];
        auto next = [&]() -> const char* {
            if (a + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", s.c_str()); std::exit(2); }
            return argv[++a];
        };
        if (s == "--problem") o.problem = next();
        else if (s == "--n") o.n = std::atoi(next());
        else if (s == "--steps") o.steps = std::atoi(next());
        else if (s == "--ts-out") o.tsOut = std::atoi(next());
        else if (s == "--prec") o.prec = std::string(next()) == "fp32flux" ? GAM_FP32FLUX : GAM_FP64;
        else if (s == "--dump") o.dump = next();
        else { std::fprintf(stderr, "unknown option %s\n", s.c_str()); std::exit(2); }
    }
    return o;
}

// Model_T defaults of the step (init.F90:312-492): the same values kaiju_b200.gamera.Model carries
gam_model_c defaultModel(int Nip, int Njp, int Nkp) {
    gam_model_c m;
    std::memset(&m, 0, sizeof m);
    m.Nip = Nip; m.Njp = Njp; m.Nkp = Nkp; m.nG = 4;
    m.gamma = 5.0 / 3.0; m.CFL = (double)0.3f; m.pdmb = 0.75; m.Vd0 = 0.5;
    m.cHogH = 0.25; m.cHogM = 0.25; m.Ca = 1.0e12; m.dFloor = 1.0e-12; m.pFloor = 1.0e-12; m.limDT0 = 1.0e-3;
    m.t = 0.0; m.tFin = 1.0e30; m.dt = 0.0; m.dt0 = 0.0; m.ts = 0;
    m.doMHD = 1; m.doBoris = 0; m.do25D = Nkp == 1; m.doLFMLim = 1; m.rmeth = GAM_RM_8CENT;
    m.bwD0 = 1.0; m.bwP0 = 0.1;
    return m;
}

// Corner index (i,j,k) counted from the first ghost of a (Ni+1)x(Nj+1)x(Nk+1)x3 Fortran array
struct Corners {
    int Ni, Nj, Nk;
    std::vector<double> xyz;
    Corners(int Nip, int Njp, int Nkp) : Ni(Nip + 8), Nj(Njp + 8), Nk(Nkp + 8),
        xyz((size_t)(Ni + 1) * (Nj + 1) * (Nk + 1) * 3) {}
    double& at(int i, int j, int k, int c) {
        return xyz[(size_t)i + (size_t)(Ni + 1) * ((size_t)j + (size_t)(Nj + 1) * ((size_t)k + (size_t)(Nk + 1) * c))];
    }
};

// Uniform Cartesian corners on [lo,hi] per axis (genGridXML, init.F90:669-731), optionally warped
// x' = x + a sin(2 pi y) sin(2 pi z) and cyclic (the warped blast-wave grid)
void cartesian(Corners& C, int Nip, int Njp, int Nkp, const double* bds, double warp) {
    double dx = (bds[1] - bds[0]) / Nip, dy = (bds[3] - bds[2]) / Njp, dz = (bds[5] - bds[4]) / Nkp;
    for (int k = 0; k <= C.Nk; ++k)
        for (int j = 0; j <= C.Nj; ++j)
            for (int i = 0; i <= C.Ni; ++i) {
                double x = bds[0] + (i - 4) * dx, y = bds[2] + (j - 4) * dy, z = bds[4] + (k - 4) * dz;
                if (warp != 0.0) {
                    double xw = x + warp * std::sin(2 * PI * y) * std::sin(2 * PI * z);
                    double yw = y + warp * std::sin(2 * PI * z) * std::sin(2 * PI * x);
                    double zw = z + warp * std::sin(2 * PI * x) * std::sin(2 * PI * y);
                    x = xw; y = yw; z = zw;
                }
                C.at(i, j, k, 0) = x; C.at(i, j, k, 1) = y; C.at(i, j, k, 2) = z;
            }
}

// LFM-type spherical corners about the x axis: r geometric, theta on [th0, pi-th0], phi periodic in k
void lfm(Corners& C, int Nip, int Njp, int Nkp, double rin, double rout, double q, double th0) {
    double dr0 = (rout - rin) * (q - 1.0) / (std::pow(q, (double)Nip) - 1.0);
    for (int k = 0; k <= C.Nk; ++k)
        for (int j = 0; j <= C.Nj; ++j)
            for (int i = 0; i <= C.Ni; ++i) {
                double r = rin + dr0 * (std::pow(q, (double)(i - 4)) - 1.0) / (q - 1.0);
                double th = th0 + (double)(j - 4) * (PI - 2.0 * th0) / Njp;
                int kk = ((k - 4) % Nkp + Nkp) % Nkp;
                double ph = (double)kk * 2.0 * PI / Nkp;
                C.at(i, j, k, 0) = r * std::cos(th);
                C.at(i, j, k, 1) = r * std::sin(th) * std::cos(ph);
                C.at(i, j, k, 2) = r * std::sin(th) * std::sin(ph);
            }
}

int check(int rc, const char* what) {
    if (rc != GAM_OK) {
        std::fprintf(stderr, "%s: %s (%d)\n", what, gam_gpu_errstr(rc), rc);
        std::exit(1);
    }
    return rc;
}

}  // namespace

int main(int argc, char** argv) {
    Opts o = parse(argc, argv);
    int Nip = o.n, Njp = o.n, Nkp = o.n, ic = GAM_IC_BW;
    gam_model_c m;
    if (o.problem == "ot") {   // Orszag-Tang 2.5D-like slab on [0,1]^2 x [0, 4/128], periodic
        Nkp = 4;
        m = defaultModel(Nip, Njp, Nkp);
        ic = GAM_IC_OT2D;
    } else if (o.problem == "lfmbw") {   // the LFM blast wave (tests/gamera/lfmbw.xml) with ring averaging
        Njp = o.n * 3 / 4; Nkp = 64;
        m = defaultModel(Nip, Njp, Nkp);
        ic = GAM_IC_LFMBW;
        m.pdmb = 1.0; m.rmeth = GAM_RM_7UP; m.dFloor = 1e-4; m.pFloor = 1e-6; m.doBoris = 1; m.Ca = 10.0;
        int bc[6] = {GAM_BC_LFMBW, GAM_BC_LFMBW, GAM_BC_LFMPOLE, GAM_BC_LFMPOLE, GAM_BC_PERIODIC, GAM_BC_PERIODIC};
        for (int n = 0; n < 6; ++n) m.bc[n] = bc[n];
        m.doRing = 1; m.ringNumR = 4; m.ringNch[0] = 8; m.ringNch[1] = 16; m.ringNch[2] = 32; m.ringNch[3] = 32;
        m.ringRecon = GAM_RING_PPM; m.ringDoS = m.ringDoE = 1; m.predFixLFM = 1; m.dtActive = 1;
    } else {   // 3D blast wave on the warped cube, zero-gradient boundaries
        m = defaultModel(Nip, Njp, Nkp);
        for (int n = 0; n < 6; ++n) m.bc[n] = GAM_BC_ZEROGRAD;
    }
    Corners C(Nip, Njp, Nkp);
    if (o.problem == "ot") {
        double b[6] = {0.0, 1.0, 0.0, 1.0, 0.0, 4.0 / 128.0};
        cartesian(C, Nip, Njp, Nkp, b, 0.0);
    } else if (o.problem == "lfmbw") {
        lfm(C, Nip, Njp, Nkp, 10.0, 100.0, 1.03, 0.05);
    } else {
        double b[6] = {-0.5, 0.5, -0.5, 0.5, -0.5, 0.5};
        cartesian(C, Nip, Njp, Nkp, b, 0.04);
    }

    gam_gpu_t* h = nullptr;
    check(gam_gpu_create_from_corners(&h, &m, C.xyz.data(), ic), "gam_gpu_create_from_corners");
    if (o.prec != GAM_FP64) check(gam_gpu_set_precision(h, o.prec), "gam_gpu_set_precision");

    // main loop: console line every tsOut steps (the reference's gamera.x cadence), one step per call
    auto w0 = std::chrono::steady_clock::now();
    double dt = 0.0, t = 0.0;
    int ts = 0;
    for (int s = 0; s < o.steps; ++s) {
        check(gam_gpu_step(h, &dt, &ts, &t), "gam_gpu_step");
        if (o.tsOut > 0 && (ts % o.tsOut == 0 || s == o.steps - 1)) {
            double divb = 0.0;
            check(gam_gpu_divb(h, &divb), "gam_gpu_divb");
            std::printf("ts = %6d  t = %.6e  dt = %.6e  divB = %.3e\n", ts, t, dt, divb);
        }
    }
    double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    if (!o.dump.empty()) {   // State%Gas after the stepped run
        size_t nc = (size_t)(Nip + 8) * (Njp + 8) * (Nkp + 8);
        std::vector<double> gas(nc * 5);
        check(gam_gpu_fetch(h, "gas", gas.data(), (long long)gas.size()), "gam_gpu_fetch");
        FILE* f = std::fopen(o.dump.c_str(), "wb");
        if (!f || std::fwrite(gas.data(), sizeof(double), gas.size(), f) != gas.size()) {
            std::fprintf(stderr, "cannot write %s\n", o.dump.c_str());
            return 1;
        }
        std::fclose(f);
    }
    // device-timed throughput: graph-replayed steps with the time step kept on the device
    double ms = 0.0;
    check(gam_gpu_run_steps_timed(h, o.steps, &ms), "gam_gpu_run_steps_timed");
    double zones = (double)Nip * Njp * Nkp;
    gam_status_c st;
    check(gam_gpu_get_status(h, &st), "gam_gpu_get_status");
    std::printf("{\"problem\": \"%s\", \"cells\": [%d, %d, %d], \"steps\": %d, \"wall_s\": %.4f, "
                "\"zone_updates_per_s_host\": %.4e, \"zone_updates_per_s_device\": %.4e, \"t\": %.6e, \"ts\": %d}\n",
                o.problem.c_str(), Nip, Njp, Nkp, o.steps, wall, zones * o.steps / wall,
                ms > 0 ? zones * o.steps / (ms * 1e-3) : 0.0, st.t, st.ts);
    gam_gpu_destroy(h);
    return 0;
}
