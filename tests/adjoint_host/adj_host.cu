// adj_host.cu -- test harness: runs the discrete-adjoint point functions of
// csrc/tns_adjoint.cuh on the host, in the order the CUDA kernels of tns_adjoint.cu run
// them, from forward values supplied by the caller.  Lets the tests compare every
// derivative with torch.autograd on a machine without a GPU.  Test infrastructure only:
// nothing in the library calls it.
#include <cstring>
#include <vector>

#include "../../2d-turbulent-navier-stokes_b200/csrc/tns_adjoint.cuh"
#include "../../2d-turbulent-navier-stokes_b200/csrc/tns_params.h"

using namespace tns;
using namespace tns::adj;

extern "C" int adj_host_step(const tns_params* prm, int ni, int nj, const double* x, const double* y,
                             const double* cfldl, const int* gtype, const int* grank, const double* gxc,
                             const double* gyc, const double* ginj, const double* q0, const double* q1, const double* q2,
                             const double* q3, const double* D, const double* VIS, const double* DT,
                             double dtmin, double* lam, int geo, double* sens) {
    AdjArgs a{};
    a.P = make_params(*prm);
    a.M.ni = ni;
    a.M.nj = nj;
    a.M.x = x;
    a.M.y = y;
    a.M.cfldl = cfldl;
    a.M.gtype = gtype;
    a.M.grank = grank;
    a.M.gxc = gxc;
    a.M.gyc = gyc;
    a.M.ginj = ginj;
    a.ni = ni;
    a.nj = nj;
    a.ncell = (long long)ni * nj;
    a.npad = (long long)(ni + 2) * (nj + 2);
    a.nnode = (long long)(ni + 1) * (nj + 1);
    a.nif = (long long)(ni + 1) * nj;
    a.njf = (long long)ni * (nj + 1);
    const long long n = a.ncell;
    std::vector<double> w(4 * NWROW * a.npad), lamA(5 * n), lamB(5 * n), lamold(5 * n), lamg(5 * n), lamd(5 * n),
        gbar(4 * 5 * a.npad, 0.0),
        srcn(16 * n), srcg(8 * n), wself(5 * n), wvisc(5 * a.npad, 0.0), dbar(5 * n), visbar(4 * n), dtbar(n),
        dpre(NDPRE * n), dout(NDOUT * n), navg(NNA * a.nnode), nbar(5 * a.nnode), vfi(NVF * a.nif),
        vfj(NVF * a.njf), xcs(a.npad), ycs(a.npad);
    const long long ng = 2LL * (ni + nj);
    std::vector<double> gport(4 * ng, 0.0), gportb(4 * ng, 0.0), portacc(3 * ng, 0.0);
    std::vector<int> ninfo(a.nnode);
    double dts = 0.0;
    a.qold = q0;
    a.d = D;
    a.vis = VIS;
    a.dt = DT;
    a.dtmin = &dtmin;
    a.w = w.data();
    a.xcs = xcs.data();
    a.ycs = ycs.data();
    a.lam_old = lamold.data();
    a.lamg = lamg.data();
    a.lamd = lamd.data();
    a.gbar4 = gbar.data();
    a.w4 = w.data();
    a.srcn = srcn.data();
    a.srcg = srcg.data();
    a.wself = wself.data();
    a.wvisc = wvisc.data();
    a.dbar = dbar.data();
    a.visbar = visbar.data();
    a.dtbar = dtbar.data();
    a.dpre = dpre.data();
    a.dout = dout.data();
    a.navg = navg.data();
    a.ninfo = ninfo.data();
    a.nbar = nbar.data();
    a.vfi = vfi.data();
    a.vfj = vfj.data();
    a.dtsum = &dts;
    a.sens = geo;
    a.geo = geo;
    a.gportb4 = gportb.data();
    a.portacc = portacc.data();
    double* sp = sens;
    a.sxbar = sp; sp += 4 * n;
    a.sybar = sp; sp += 4 * n;
    a.volbar = sp; sp += n;
    a.dlbar = sp; sp += n;
    a.xcbar = sp; sp += a.npad;
    a.ycbar = sp; sp += a.npad;
    a.xnbar = sp; sp += a.nnode;
    a.ynbar = sp; sp += a.nnode;
    a.rtolc = sp; sp += n;
    a.rtoln = sp; sp += a.nnode;
    a.t0bar = sp; sp += n;
    a.s0bar = sp;
    for (long long p = 0; p < a.npad; p++) centroid_point(a, p);
    const double alpha[4] = {0.25, 1.0 / 3.0, 0.5, 1.0};
    const double* qs[4] = {q0, q1, q2, q3};
    for (int k = 0; k < 4; k++) {
        a.qst[k] = qs[k];
        for (long long g = 0; g < ng; g++) gport_point(a, g, qs[k], gport.data() + k * ng);
    }
    double* lam_stage[5] = {nullptr, lamA.data(), lamB.data(), lamA.data(), lam};  // adjoint of Q_k
    for (int st = 3; st >= 0; st--) {
        a.qin = qs[st];
        a.alpha = alpha[st];
        a.first = st == 3;
        a.stage1 = st == 0;
        a.lam_in = lam_stage[st + 1];
        a.lam_out = lam_stage[st];
        a.w = w.data() + (size_t)st * NWROW * a.npad;
        a.gbar = gbar.data() + (size_t)st * 5 * a.npad;
        a.gport = gport.data() + st * ng;
        a.gportb = gportb.data() + st * ng;
        for (long long p = 0; p < a.npad; p++) s0_point(a, p);
        for (long long c = 0; c < n; c++) s1_point(a, c);
        if (st == 0) {
            for (long long k = 0; k < a.nnode; k++) v0_point(a, k);
            for (long long f = 0; f < a.nif + a.njf; f++) v1_point(a, f);
            for (long long k = 0; k < a.nnode; k++) v2_point(a, k);
            for (long long p = 0; p < a.npad; p++) v3_point(a, p);
        }
        for (long long c = 0; c < n; c++) s3_point(a, c);
        for (long long c = 0; c < band_count(a); c++) s3g_point(a, c);
        for (long long c = 0; c < n; c++) port_point(a, c);
    }
    if (geo) {
        for (long long c = 0; c < n; c++) geo_point(a, c);
        for (long long k = 0; k < a.nnode; k++) port_node_point(a, k);
    }
    for (long long c = 0; c < n; c++) d0_point(a, c);
    for (long long c = 0; c < n; c++) d1_point(a, c);
    for (long long c = 0; c < n; c++) d2_point(a, c);
    if (!a.P.local) {
        for (long long c = 0; c < n; c++) dts += dtbar[c];
        for (long long c = 0; c < n; c++) dtmin_point(a, c);
    }
    a.lam_out = lam;
    for (long long c = 0; c < n; c++) final_point(a, c);
    return 0;
}
