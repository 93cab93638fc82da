// tnsmain.cpp -- the solver's main program (twodturb / axiturb) with the RK4 loop on the
// GPU.  It keeps the reference main's file behaviour (src/solvers/turbnstwod.f90; the
// axisymmetric turbnsaxis.f90 is identical): it reads flow.in, grid.in, bc.in (and
// restart.in when ISTART=1) from the working directory, prints the CDIFF monitor every
// 1000 iterations and appends it to fort.32, writes restartNNNNNNNNNN.in every 20000
// iterations, and restart.in and tec_plot.dat at the end.  The hot loop runs through the
// C ABI of include/tnsgpu.h.
//
// Inputs the reference declares but never assigns (BC types 6 and 7) come from an
// optional file `bc67.in`: TFLAME ANCOMB ACOMB RHOPROP PINF AMINF DELTABL on one line,
// and an optional `injection.in` with one burn-rate multiplier per bc.in line.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/tnsgpu.h"

#ifndef TNS_DEFAULT_IAXIS
#define TNS_DEFAULT_IAXIS 0
#endif

namespace {

// Fortran list-directed input: each READ starts at a new record and takes whitespace- or
// comma-separated values, continuing onto further records when one runs short.
struct ListReader {
    std::ifstream in;
    std::string name;
    explicit ListReader(const std::string& path) : in(path), name(path) {}
    bool ok() const { return (bool)in; }
    std::vector<std::string> read(size_t n) {
        std::vector<std::string> tok;
        std::string line;
        while (tok.size() < n && std::getline(in, line)) {
            for (char& c : line)
                if (c == ',' || c == '\t' || c == '\r') c = ' ';
            std::istringstream ss(line);
            std::string t;
            while (tok.size() < n && ss >> t) tok.push_back(t);
        }
        if (tok.size() < n) {
            std::fprintf(stderr, "%s: end of file while reading %zu values\n", name.c_str(), n);
            std::exit(2);
        }
        return tok;
    }
};

double num(const std::string& s) {
    std::string t = s;
    for (char& c : t)
        if (c == 'd' || c == 'D') c = 'e';  // Fortran 1.0D0
    return std::strtod(t.c_str(), nullptr);
}

// Fortran Ew.d edit descriptor (0.ddddddE+xx).
std::string fortran_e(double v, int w, int d) {
    char buf[64];
    if (!std::isfinite(v)) {
        std::snprintf(buf, sizeof buf, "%*s", w, std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity"));
        return buf;
    }
    int e = 0;
    double m = std::fabs(v);
    if (m != 0.0) {
        e = (int)std::floor(std::log10(m)) + 1;
        m = m / std::pow(10.0, e);
        double scaled = std::nearbyint(m * std::pow(10.0, d));
        if (scaled >= std::pow(10.0, d)) { e += 1; scaled = std::nearbyint(scaled / 10.0); }
        if (scaled < std::pow(10.0, d - 1)) { e -= 1; scaled *= 10.0; }
        m = scaled;
    }
    std::string digits;
    {
        char db[64];
        std::snprintf(db, sizeof db, "%0*.0f", d, m);
        digits = db;
    }
    char eb[16];
    std::snprintf(eb, sizeof eb, "E%c%02d", e < 0 ? '-' : '+', std::abs(e));
    std::string body = "0." + digits + eb;
    if (v < 0) body = "-" + body;
    if ((int)body.size() > w && body.compare(0, 2, "0.") == 0) body.erase(0, 1);
    if ((int)body.size() > w && body.compare(0, 3, "-0.") == 0) body.erase(1, 1);
    if ((int)body.size() < w) body = std::string(w - body.size(), ' ') + body;
    return body;
}

// List-directed output of one REAL(8) (round-trips exactly).
std::string ld(double v) {
    char buf[40];
    std::snprintf(buf, sizeof buf, "  %24.17E", v);
    return buf;
}

void die(tns_handle* h, int rc, const char* what) {
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, h ? tns_last_error(h) : "");
    std::exit(1);
}

}  // namespace

int main() {
    // flow.in (turbnstwod.f90:20-23)
    ListReader flow("flow.in");
    if (!flow.ok()) { std::fprintf(stderr, "cannot open flow.in\n"); return 2; }
    auto f = flow.read(17);
    const std::string fnamegrid = f[0], fnamebc = f[1];
    tns_params P{};
    P.gama = num(f[2]); P.amol = num(f[3]);
    P.local = (int)num(f[4]);
    const long long niter = (long long)num(f[5]);
    const int istart = (int)num(f[6]);
    P.cfl = num(f[7]); P.prandtl = num(f[8]); P.prandtlt = num(f[9]);
    P.p0 = num(f[10]); P.t0 = num(f[11]); P.pamb = num(f[12]);
    const double amachinit = num(f[13]);
    P.rtred = num(f[14]);
    P.npseudo = (int)num(f[15]);
    P.iaxis = f.size() > 16 ? (int)num(f[16]) : TNS_DEFAULT_IAXIS;
    P.precision = 0;
    {
        ListReader x("bc67.in");
        if (x.ok()) {
            auto t = x.read(7);
            P.tflame = num(t[0]); P.ancomb = num(t[1]); P.acomb = num(t[2]); P.rhoprop = num(t[3]);
            P.pinf = num(t[4]); P.aminf = num(t[5]); P.deltabl = num(t[6]);
        }
    }

    // grid.in and bc.in (geometry.f90:31-52); coordinates scaled by MM_TO_M
    ListReader grid(fnamegrid);
    if (!grid.ok()) { std::fprintf(stderr, "cannot open %s\n", fnamegrid.c_str()); return 2; }
    auto h0 = grid.read(2);
    const int nods = (int)num(h0[0]), neles = (int)num(h0[1]);
    std::vector<double> X(nods + 1, 0.0), Y(nods + 1, 0.0);
    for (int i = 0; i < nods; i++) {
        auto t = grid.read(3);
        const int n = (int)num(t[0]);
        if (n < 1 || n > nods) { std::fprintf(stderr, "%s: node id %d out of range\n", fnamegrid.c_str(), n); return 2; }
        X[n] = num(t[1]) * 0.001;
        Y[n] = num(t[2]) * 0.001;
    }
    std::vector<int> NOD(4 * (size_t)neles), NC[4];
    for (auto& v : NC) v.resize(neles);
    for (int i = 0; i < neles; i++) {
        auto t = grid.read(9);
        for (int k = 0; k < 4; k++) NOD[(size_t)k * neles + i] = (int)num(t[1 + k]);
        for (int k = 0; k < 4; k++) NC[k][i] = (int)num(t[5 + k]);
    }
    ListReader bc(fnamebc);
    if (!bc.ok()) { std::fprintf(stderr, "cannot open %s\n", fnamebc.c_str()); return 2; }
    const int nghosts = (int)num(bc.read(1)[0]);
    std::vector<int> NPARENT(nghosts), NGHOST(nghosts), NTYPE(nghosts), NSIDE(nghosts);
    for (int i = 0; i < nghosts; i++) {
        auto t = bc.read(4);
        NPARENT[i] = (int)num(t[0]); NGHOST[i] = (int)num(t[1]);
        NTYPE[i] = (int)num(t[2]); NSIDE[i] = (int)num(t[3]);
    }

    // thermodynamics and initial state (turbnstwod.f90:37-90)
    const double RR = 8314.0 / P.amol, CV = RR / (P.gama - 1.0);
    std::vector<double> C[5];
    for (auto& v : C) v.assign(neles, 0.0);
    double RINIT = 0.0;
    long long niterold = 0;
    if (istart == 0) {
        const double dyn = 1.0 + (P.gama - 1.0) * 0.5 * std::pow(amachinit, 2.0);
        const double tinit = P.t0 / dyn;
        const double pinit = P.p0 / std::pow(dyn, P.gama / (P.gama - 1.0));
        const double uinit = amachinit * std::sqrt(P.gama * RR * tinit);
        const double vinit = 0.0;
        const double einit = CV * tinit + 0.5 * (std::pow(uinit, 2.0) + std::pow(vinit, 2.0));
        const double rhoinit = pinit / (RR * tinit);
        const double amuinit = (0.00000011848) * std::sqrt(P.amol) * std::pow(tinit, 0.6);
        RINIT = amuinit / rhoinit;
        for (int i = 0; i < neles; i++) {
            C[0][i] = rhoinit; C[1][i] = rhoinit * uinit; C[2][i] = rhoinit * vinit;
            C[3][i] = rhoinit * einit; C[4][i] = rhoinit * RINIT;
        }
    } else {
        ListReader rs("restart.in");
        if (!rs.ok()) { std::fprintf(stderr, "cannot open restart.in\n"); return 2; }
        for (int i = 0; i < neles; i++) {
            auto t = rs.read(5);
            for (int k = 0; k < 5; k++) C[k][i] = num(t[k]);
        }
        P.rtred = num(rs.read(1)[0]);
        P.npseudo = (int)num(rs.read(1)[0]);
        RINIT = num(rs.read(1)[0]);
        niterold = (long long)num(rs.read(1)[0]);
    }
    P.rinit = RINIT;

    tns_mesh M{};
    M.nods = nods; M.neles = neles; M.nghosts = nghosts;
    M.x = X.data() + 1; M.y = Y.data() + 1;
    M.nod = NOD.data(); M.ld_nod = neles;
    M.nc1 = NC[0].data(); M.nc2 = NC[1].data(); M.nc3 = NC[2].data(); M.nc4 = NC[3].data();
    M.nparent = NPARENT.data(); M.nghost = NGHOST.data(); M.ntype = NTYPE.data(); M.nside = NSIDE.data();
    tns_handle* h = nullptr;
    int rc = tns_create(&M, &P, &h);
    if (rc) die(h, rc, "tns_create");
    {
        ListReader inj("injection.in");
        if (inj.ok()) {
            auto t = inj.read(nghosts);
            std::vector<double> s(nghosts);
            for (int i = 0; i < nghosts; i++) s[i] = num(t[i]);
            if ((rc = tns_set_injection_scale(h, s.data()))) die(h, rc, "tns_set_injection_scale");
        }
    }
    if ((rc = tns_upload_state(h, C[0].data(), C[1].data(), C[2].data(), C[3].data(), C[4].data())))
        die(h, rc, "tns_upload_state");

    auto write_restart = [&](const char* path, long long count) {
        FILE* fp = std::fopen(path, "w");
        if (!fp) { std::fprintf(stderr, "cannot write %s\n", path); std::exit(2); }
        for (int i = 0; i < neles; i++)
            std::fprintf(fp, "%s%s%s%s%s\n", ld(C[0][i]).c_str(), ld(C[1][i]).c_str(), ld(C[2][i]).c_str(),
                         ld(C[3][i]).c_str(), ld(C[4][i]).c_str());
        std::fprintf(fp, "%s\n %11d\n%s\n %11lld\n", ld(P.rtred).c_str(), P.npseudo, ld(RINIT).c_str(), count);
        std::fclose(fp);
    };

    // the RK4 loop (turbnstwod.f90:95-183) in chunks ending at monitor / restart points
    FILE* f32 = std::fopen("fort.32", "w");
    long long it = 0;
    while (it < niter) {
        long long next = niter;
        const long long nmon = (it / 1000 + 1) * 1000;
        const long long nrst = ((niterold + it) / 20000 + 1) * 20000 - niterold;
        if (nmon < next) next = nmon;
        if (nrst < next) next = nrst;
        const int chunk = (int)(next - it);
        double cd[5];
        int nrec = 0;
        // the monitor fires on the chunk's last iteration exactly when it is a multiple of 1000
        const bool mon = next % 1000 == 0;
        if ((rc = tns_run(h, chunk, mon ? chunk : 0, cd, 1, &nrec))) die(h, rc, "tns_run");
        it = next;
        if (mon && nrec == 1) {
            std::printf("%10lld", it + niterold);
            for (int k = 0; k < 5; k++) std::printf("     %s", fortran_e(cd[k], 12, 6).c_str());
            std::printf("\n");
            if (f32) {
                for (int k = 0; k < 5; k++) std::fprintf(f32, "%s", fortran_e(cd[k], 15, 5).c_str());
                std::fprintf(f32, "\n");
            }
        }
        if ((niterold + it) % 20000 == 0) {
            if ((rc = tns_download_state(h, C[0].data(), C[1].data(), C[2].data(), C[3].data(), C[4].data())))
                die(h, rc, "tns_download_state");
            char name[32];
            std::snprintf(name, sizeof name, "restart%10lld.in", niterold + it);
            write_restart(name, niterold + it);
        }
    }
    if (f32) std::fclose(f32);
    if ((rc = tns_download_state(h, C[0].data(), C[1].data(), C[2].data(), C[3].data(), C[4].data())))
        die(h, rc, "tns_download_state");
    write_restart("restart.in", niterold + niter);

    // POSTPROCESS (solver_state.f90:230-283)
    std::printf(" Postprocessing.\n  \n");
    if (niter > 0) {
        // node averages of P, U, V, T computed on the GPU (tns_node_averages)
        std::vector<double> s1(nods + 1, 0.0), s2(nods + 1, 0.0), s3(nods + 1, 0.0), s4(nods + 1, 0.0);
        if ((rc = tns_node_averages(h, s1.data() + 1, s2.data() + 1, s3.data() + 1, s4.data() + 1)))
            die(h, rc, "tns_node_averages");
        FILE* tp = std::fopen("tec_plot.dat", "w");
        std::fprintf(tp, " VARIABLES = \"X\", \"Y\", \"U\", \"V\", \"P\", \"RHO\", \"MACH\", \"T\"\n");
        std::fprintf(tp, " ZONE F = FEPOINT, ET = QUADRILATERAL, N = %12d , E = %12d\n", nods, neles);
        for (int i = 1; i <= nods; i++) {
            const double PNN = s1[i], UNN = s2[i], VNN = s3[i], TNN = s4[i];
            const double AMN = std::sqrt(UNN * UNN + VNN * VNN) / std::sqrt(P.gama * RR * TNN);
            const double RON = PNN / (RR * TNN);
            std::fprintf(tp, "%s%s%s%s%s%s%s%s\n", ld(X[i]).c_str(), ld(Y[i]).c_str(), ld(UNN).c_str(),
                         ld(VNN).c_str(), ld(PNN * 0.00001).c_str(), ld(RON).c_str(), ld(AMN).c_str(),
                         ld(TNN).c_str());
        }
        for (int i = 0; i < neles; i++)
            std::fprintf(tp, " %11d %11d %11d %11d\n", NOD[i], NOD[(size_t)neles + i],
                         NOD[2 * (size_t)neles + i], NOD[3 * (size_t)neles + i]);
        std::fclose(tp);
    }
    tns_destroy(h);
    return 0;
}
