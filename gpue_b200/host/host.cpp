// host.cpp -- GPUE's command line, init(), file formats and the evolve()
// shim over the C ABI (see host.h for the reference interfaces).

#include "host.h"

#include <getopt.h>
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>

namespace gpue_host {

namespace {

const double kPI = 3.141592653589793;   // include/constants.h
const double kHBAR = 1.05457148e-34;    // include/constants.h
const double kMass = 1.4431607e-25;     // Rb-87, src/init.cu:98
const double kAs = 4.76e-9;             // src/init.cu:100

void check(gpue_status st, const gpue_ctx* c, const char* what) {
    if (st == GPUE_OK) return;
    std::ostringstream o;
    o << what << " failed (status " << (int)st << ")";
    const char* msg = c ? gpue_last_error(c) : "";
    if (msg && *msg) o << ": " << msg;
    throw std::runtime_error(o.str());
}

bool file_exists(const std::string& f) {
    struct stat st;
    return stat(f.c_str(), &st) == 0;
}

std::string filecheck(const std::string& f) {
    if (!file_exists(f)) throw std::runtime_error("file " + f + " not found");
    return f;
}

// Position of flat index g = i + xDim*(j + yDim*k) (x fastest).
struct Point {
    double x, y, z;
};
Point point(const Grid& par, size_t g) {
    const size_t nx = par.ival("xDim"), ny = par.ival("yDim");
    return {par.x[g % nx], par.y[(g / nx) % ny], par.z[g / (nx * ny)]};
}

// Full-field Ax, Ay, Az for the gauge of -A (Grid::set_A_fn, src/ds.cu:300-331;
// generate_gauge, src/operators.cu:471-615): the field kernels of
// src/operators.cu:621-720 evaluated on the host, or file_A
// (src/operators.cu:259-270) for -A file.  In 2D, Az is zero and the presets
// see zMax = 1 (generate_gauge's default).
void gauge_tables(const Grid& par, std::vector<double> (&A)[3]) {
    const int dimnum = par.ival("dimnum");
    const size_t n = (size_t)par.ival("xDim") * par.ival("yDim") * par.ival("zDim");
    for (auto& a : A) a.assign(n, 0.0);
    const double omega = par.dval("omega"), omegaX = par.dval("omegaX"),
                 omegaY = par.dval("omegaY");
    const double xMax = par.dval("xMax"), yMax = par.dval("yMax");
    const double zMax = dimnum == 3 ? par.dval("zMax") : 1.0;
    if (par.Afn == "file") {
        const char* keys[3] = {"Axfile", "Ayfile", "Azfile"};
        for (int a = 0; a < (dimnum == 3 ? 3 : 2); ++a) {
            std::ifstream in(par.sval(keys[a]));
            std::vector<double> v;
            double t;
            while (in >> t) v.push_back(omega * t);
            if (v.size() != n)
                throw std::runtime_error(par.sval(keys[a]) + " has " + std::to_string(v.size()) +
                                         " values, the grid " + std::to_string(n));
            A[a] = v;
        }
        return;
    }
    for (size_t g = 0; g < n; ++g) {
        const Point q = point(par, g);
        if (par.Afn == "rotation") {  // krotation_Ax / krotation_Ay
            A[0][g] = -q.y * omega * omegaX;
            A[1][g] = q.x * omega * omegaY;
        } else if (par.Afn == "ring_rotation") {  // kring_rotation_A{x,y,z}
            const double theta = std::atan2(q.y, q.x);
            A[0][g] = (q.z + zMax) * std::cos(theta) * omega * omegaX;
            A[1][g] = (q.z + zMax) * std::sin(theta) * omega * omegaX;
            if (dimnum == 3) A[2][g] = std::sqrt(q.x * q.x + q.y * q.y) * omega * omegaX;
        } else if (par.Afn == "ring") {  // kring_Az
            const double rad = std::sqrt(q.x * q.x + q.y * q.y);
            if (dimnum == 3) A[2][g] = omega * std::exp(-rad * rad / (0.0001 * xMax)) * 0.01;
        } else if (par.Afn == "test") {  // ktest_Ax
            A[0][g] = (std::sin(q.y * 100000) + 1) * yMax * omega;
        }
    }
}

// ktorus_V (src/operators.cu:1011-1029) with GPUE's items array
// (src/operators.cu:753-792): omegaZ and z0_shift only in 3D.
std::vector<double> torus_V(const Grid& par, const std::vector<double> (&A)[3]) {
    const int dimnum = par.ival("dimnum");
    const size_t n = A[0].size();
    const double xMax = par.dval("xMax"), omegaX = par.dval("omegaX"),
                 omegaY = par.dval("omegaY"), mass = par.dval("mass"),
                 fudge = par.dval("fudge");
    const double omegaZ = dimnum == 3 ? par.dval("omegaZ") : 0.0;
    const double x0 = par.dval("x0_shift"), y0 = par.dval("y0_shift");
    const double z0 = dimnum == 3 ? par.dval("z0_shift") : 0.0;
    std::vector<double> V(n);
    for (size_t g = 0; g < n; ++g) {
        const Point q = point(par, g);
        const double rad = std::sqrt((q.x - x0) * (q.x - x0) + (q.y - y0) * (q.y - y0)) -
                           0.5 * xMax;
        const double omegaR = omegaX * omegaX + omegaY * omegaY;
        const double V_tot = 2 * omegaZ * omegaZ * (q.z - z0) * (q.z - z0) +
                             omegaR * (rad * rad + fudge * rad * q.z);
        V[g] = 0.5 * mass * (V_tot + A[0][g] * A[0][g] + A[1][g] * A[1][g] + A[2][g] * A[2][g]);
    }
    return V;
}

// The context of this Grid, created on first use from its keys; a
// parameter file (-I) is loaded into it with the Grid's doubles as names.
gpue_ctx* ensure_ctx(Grid& par) {
    if (par.ctx()) return par.ctx();
    gpue_params p = params_from_grid(par);
    gpue_ctx* c = nullptr;
    check(gpue_ctx_create(&p, &c), nullptr, "gpue_ctx_create");
    par.set_ctx(c);
    if (par.bval("use_param_file")) {
        std::ifstream f(par.sval("param_file"));
        std::stringstream text;
        text << f.rdbuf();
        static const char* keys[] = {"omega", "omegaX", "omegaY", "omegaZ", "gammaY", "xMax",
                                     "yMax", "zMax", "dx", "dy", "dz", "mass", "a_s",
                                     "interaction", "gDenConst", "x0_shift", "y0_shift",
                                     "z0_shift", "Rxy", "a0x", "a0y", "a0z", "winding",
                                     "fudge", "dt", "gdt"};
        std::vector<const char*> names;
        std::vector<double> values;
        for (const char* k : keys)
            if (par.has(k)) {
                names.push_back(k);
                values.push_back(par.dval(k));
            }
        check(gpue_load_param_text(c, text.str().c_str(), 0, names.data(), values.data(),
                                   (int32_t)names.size()),
              c, "parameter file");
    }
    const bool table_a = par.Afn == "file" || par.Afn == "ring_rotation" ||
                         par.Afn == "ring" || par.Afn == "test";
    if (table_a || par.Vfn == "torus") {
        if (par.bval("use_param_file"))
            throw std::runtime_error("-A " + par.Afn + " / -v " + par.Vfn +
                                     " tables are not combined with a parameter file");
        std::vector<double> A[3];
        gauge_tables(par, A);
        if (table_a)
            check(gpue_set_gauge_tables(c, A[0].data(), A[1].data(),
                                        par.ival("dimnum") == 3 ? A[2].data() : nullptr),
                  c, "gauge tables");
        if (par.Vfn == "torus") {
            const std::vector<double> V = torus_V(par, A);
            check(gpue_set_potential_table(c, V.data()), c, "torus potential");
        }
    }
    if (par.bval("autotune")) check(gpue_autotune(c, 0), c, "gpue_autotune");
    return c;
}

}  // namespace

void Grid::write(const std::string& file) const {
    std::ofstream out(file);
    out << "[Params]\n";
    for (const auto& kv : doubles_) out << kv.first << "=" << kv.second << '\n';
    for (const auto& kv : ints_) out << kv.first << "=" << kv.second << '\n';
}

// ------------------------------------------------------------ parseArgs --

Grid parse_args(int argc, char** argv) {
    Grid par;
    // defaults (src/parser.cu:14-67)
    par.store("xDim", 256);
    par.store("yDim", 256);
    par.store("zDim", 256);
    par.store("omega", 0.0);
    par.store("gammaY", 1.0);
    par.store("gsteps", 1);
    par.store("esteps", 1);
    par.store("gdt", 1e-4);
    par.store("dt", 1e-4);
    par.store("device", 0);
    par.store("atoms", 1);
    par.store("read_wfc", false);
    par.store("printSteps", 100);
    par.store("winding", 0.0);
    par.store("corotating", false);
    par.store("gpe", false);
    par.store("omegaZ", 6.283);
    par.store("interaction", 1.0);
    par.store("laser_power", 0.0);
    par.store("angle_sweep", 0.0);
    par.store("kick_it", 0);
    par.store("write_it", false);
    par.store("x0_shift", 0.0);
    par.store("y0_shift", 0.0);
    par.store("z0_shift", 0.0);
    par.store("sepMinEpsilon", 0.0);
    par.store("graph", false);
    par.store("unit_test", false);
    par.store("omegaX", 6.283);
    par.store("omegaY", 6.283);
    par.store("data_dir", "data/");
    par.store("ramp", false);
    par.store("ramp_type", 1);
    par.store("dimnum", 2);
    par.store("write_file", true);
    par.store("fudge", 0.0);
    par.store("kill_idx", -1);
    par.store("mask_2d", 0.0);
    par.store("box_size", -0.01);
    par.store("found_sobel", false);
    par.store("energy_calc", false);
    par.store("energy_calc_steps", 0);
    par.store("energy_calc_threshold", -1.0);
    par.store("use_param_file", false);
    par.store("param_file", "param.cfg");
    par.store("cyl_coord", false);
    par.store("conv_type", "FFT");
    par.store("charge", 0);
    par.store("flip", false);
    par.store("thresh_const", 1.0);
    // this build's options
    par.store("precision", (int)GPUE_PREC_FP64);
    par.store("autotune", false);
    par.store("print_params", false);
    par.store("checkpoint_every", 0);
    par.store("resume", false);
    par.store("start_step", 0);

    // long options first; the rest go to getopt as GPUE parses them
    std::vector<char*> args;
    args.push_back(argv[0]);
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--precision=fp32") par.store("precision", (int)GPUE_PREC_FP32);
        else if (a == "--precision=fp64") par.store("precision", (int)GPUE_PREC_FP64);
        else if (a == "--autotune") par.store("autotune", true);
        else if (a == "--print-params") par.store("print_params", true);
        else if (a.rfind("--checkpoint-every=", 0) == 0)
            par.store("checkpoint_every", std::atoi(a.c_str() + 19));
        else if (a == "--resume") par.store("resume", true);
        else if (a.rfind("--", 0) == 0) throw std::runtime_error("unknown option " + a);
        else args.push_back(argv[i]);
    }
    int ac = (int)args.size();
    args.push_back(nullptr);
    char** av = args.data();

    optind = 1;
    int opt;
    while ((opt = getopt(ac, av,
                         "b:d:D:C:x:y:w:m:G:g:e:T:t:n:p:rQ:L:E::lsi:P:X:Y:O:k:WU:V:S:ahz:H:uA:v:"
                         "Z:fc:F:K:R:q:I:j:J")) != -1) {
        switch (opt) {
            case 'x': par.store("xDim", atoi(optarg)); break;
            case 'y': par.store("yDim", atoi(optarg)); break;
            case 'z': par.store("zDim", atoi(optarg)); break;
            case 'b': par.store("box_size", atof(optarg)); break;
            case 'j': par.store("thresh_const", atof(optarg)); break;
            case 'w': par.store("omega", atof(optarg)); break;
            case 'm': par.store("mask_2d", atof(optarg)); break;
            case 'G': par.store("gammaY", atof(optarg)); break;
            case 'g': par.store("gsteps", (int)atof(optarg)); break;
            case 'e': par.store("esteps", (int)atof(optarg)); break;
            case 'F': par.store("fudge", atof(optarg)); break;
            case 'T': par.store("gdt", atof(optarg)); break;
            case 't': par.store("dt", atof(optarg)); break;
            case 'C': par.store("device", atoi(optarg)); break;
            case 'n': par.store("atoms", (int)atof(optarg)); break;
            case 'I':
                par.store("param_file", std::string(optarg));
                par.store("use_param_file", true);
                break;
            case 'R':
                par.store("ramp", true);
                par.store("ramp_type", atoi(optarg));
                break;
            case 'r': par.store("read_wfc", true); break;
            case 'p': par.store("printSteps", atoi(optarg)); break;
            case 'L': par.store("winding", atof(optarg)); break;
            case 'l': par.store("corotating", true); break;
            case 'E':
                // -E <threshold> <steps> (src/parser.cu:222-238)
                if (optind < ac && av[optind][0] != '-') {
                    par.store("energy_calc_threshold", atof(av[optind]));
                    if (optind + 1 < ac) par.store("energy_calc_steps", atoi(av[optind + 1]));
                    optind += (optind + 1 < ac && av[optind + 1][0] != '-') ? 2 : 1;
                }
                par.store("energy_calc", true);
                break;
            case 'f': par.store("write_file", false); break;
            case 'J': par.store("cyl_coord", true); break;
            case 'q':
                par.store("flip", true);
                par.store("charge", atoi(optarg));
                break;
            case 's': par.store("gpe", true); break;
            case 'Z': par.store("omegaZ", atof(optarg)); break;
            case 'i': par.store("interaction", atof(optarg)); break;
            case 'P': par.store("laser_power", atof(optarg)); break;
            case 'X': par.store("omegaX", atof(optarg)); break;
            case 'Y': par.store("omegaY", atof(optarg)); break;
            case 'O': par.store("angle_sweep", atof(optarg)); break;
            case 'k': par.store("kick_it", atoi(optarg)); break;
            case 'W': par.store("write_it", true); break;
            case 'd': par.store("data_dir", std::string(optarg) + "/"); break;
            case 'U': par.store("x0_shift", atof(optarg)); break;
            case 'V': par.store("y0_shift", atof(optarg)); break;
            case 'Q': par.store("z0_shift", atof(optarg)); break;
            case 'S': par.store("sepMinEpsilon", atof(optarg)); break;
            case 'v':
                par.Vfn = optarg;
                par.Wfcfn = optarg;
                break;
            case 'c': {
                const int dimnum = atoi(optarg);
                if (dimnum == 3) {
                    par.Kfn = "rotation_K3d";
                    par.Vfn = "3d";
                    par.Wfcfn = "3d";
                    par.store("box_size", 2.5e-5);
                }
                par.store("dimnum", dimnum);
                break;
            }
            case 'A': par.Afn = optarg; break;
            case 'a': par.store("graph", true); break;
            case 'K': par.store("kill_idx", atoi(optarg)); break;
            case 'h':
            case 'H':
            case 'u':
                throw std::runtime_error(std::string("option -") + (char)opt +
                                         " (help / unit tests) is not part of this build");
            default:
                throw std::runtime_error("unknown option");
        }
    }

    const std::string data_dir = par.sval("data_dir");
    mkdir(data_dir.c_str(), 0700);
    if (par.ival("dimnum") < 3) par.store("zDim", 1);
    if (par.ival("dimnum") < 2) par.store("yDim", 1);
    if (par.bval("use_param_file"))
        par.store("param_file", filecheck(data_dir + par.sval("param_file")));
    if (par.bval("read_wfc")) {
        par.store("infile", filecheck(data_dir + "wfc_load"));
        par.store("infilei", filecheck(data_dir + "wfci_load"));
    }
    if (par.Afn == "file") {  // src/parser.cu:478-487
        par.store("Axfile", filecheck(data_dir + "Axgauge"));
        par.store("Ayfile", filecheck(data_dir + "Aygauge"));
        if (par.ival("dimnum") == 3) par.store("Azfile", filecheck(data_dir + "Azgauge"));
    }
    return par;
}

// ----------------------------------------------------------------- init --

void init(Grid& par) {
    const int dimnum = par.ival("dimnum");
    if (dimnum != 2 && dimnum != 3)
        throw std::runtime_error("this build runs 2D and 3D grids (-c 2 or -c 3)");
    static const char* gauges[] = {"rotation", "constant", "file", "ring_rotation", "ring",
                                   "test"};
    if (std::find(std::begin(gauges), std::end(gauges), par.Afn) == std::end(gauges))
        throw std::runtime_error("gauge field '" + par.Afn +
                                 "' is not one of rotation, constant, file, ring_rotation, "
                                 "ring, test");
    if (par.Vfn != "2d" && par.Vfn != "3d" && par.Vfn != "torus")
        throw std::runtime_error("potential '" + par.Vfn + "' is not one of 2d, 3d, torus");
    const int N = par.ival("atoms");
    const int xDim = par.ival("xDim"), yDim = par.ival("yDim"), zDim = par.ival("zDim");
    const double omegaX = par.dval("omegaX"), omegaY = par.dval("omegaY"),
                 omegaZ = par.dval("omegaZ");
    const double box_size = par.dval("box_size");

    par.store("mass", kMass);
    par.store("a_s", kAs);
    const double a0x = std::sqrt(kHBAR / (2 * kMass * omegaX));
    const double a0y = std::sqrt(kHBAR / (2 * kMass * omegaY));
    const double a0z = std::sqrt(kHBAR / (2 * kMass * omegaZ));
    par.store("a0x", a0x);
    par.store("a0y", a0y);
    par.store("a0z", a0z);
    double gDenConst = N * 4 * kHBAR * kHBAR * kPI * (kAs / kMass);
    if (dimnum == 2) gDenConst *= std::sqrt(kMass * omegaZ / (2 * kPI * kHBAR));
    par.store("gDenConst", gDenConst);
    const double Rxy = std::pow(15, 0.2) * std::pow(N * kAs * std::sqrt(kMass * omegaZ / kHBAR), 0.2);
    par.store("Rxy", Rxy);
    double xMax, yMax, zMax;
    if (box_size > 0) {
        xMax = yMax = zMax = box_size;
    } else {
        xMax = 6 * Rxy * a0x;
        yMax = 6 * Rxy * a0y;
        zMax = 6 * Rxy * a0z;
    }
    par.store("xMax", xMax);
    par.store("yMax", yMax);
    par.store("zMax", zMax);
    par.store("pxMax", (kPI / xMax) * (xDim >> 1));
    par.store("pyMax", (kPI / yMax) * (yDim >> 1));
    par.store("pzMax", (kPI / zMax) * (zDim >> 1));
    const double dx = xMax / (xDim >> 1);
    const double dy = dimnum > 1 ? yMax / (yDim >> 1) : 1.0;
    const double dz = dimnum > 2 ? zMax / (zDim >> 1) : 1.0;
    par.store("dx", dx);
    par.store("dy", dy);
    par.store("dz", dz);
    par.store("dpx", kPI / xMax);
    par.store("dpy", kPI / yMax);
    par.store("dpz", kPI / zMax);
    par.store("gSize", xDim * yDim * zDim);

    // positions (generate_p_space, src/operators.cu:277-432)
    auto axis = [](int n, double xmax, double d, bool on) {
        std::vector<double> v(n, 0.0);
        if (on)
            for (int i = 0; i < n / 2; ++i) {
                v[i] = -xmax + i * d;
                v[i + n / 2] = i * d;
            }
        return v;
    };
    par.x = axis(xDim, xMax, dx, true);
    par.y = axis(yDim, yMax, dy, dimnum > 1);
    par.z = axis(zDim, zMax, dz, dimnum > 2);

    const size_t gSize = (size_t)xDim * yDim * zDim;
    if (!par.bval("read_wfc")) {
        // kstd_wfc (src/operators.cu:1031-1050), then init()'s normalisation
        // by sqrt(sum |psi| dV) -- the modulus, not its square (src/init.cu:
        // 227-230, 297-303)
        const double winding = par.dval("winding");
        par.wfc.assign(gSize, 0.0);
        double sum = 0.0;
        for (int k = 0; k < zDim; ++k)
            for (int j = 0; j < yDim; ++j)
                for (int i = 0; i < xDim; ++i) {
                    const size_t g = i + (size_t)xDim * (j + (size_t)yDim * k);
                    if (par.Wfcfn == "torus") {
                        // ktorus_wfc (src/operators.cu:1052-1067)
                        const double x0 = par.dval("x0_shift"), y0 = par.dval("y0_shift");
                        const double rad = std::sqrt((par.x[i] - x0) * (par.x[i] - x0) +
                                                     (par.y[j] - y0) * (par.y[j] - y0)) -
                                           0.5 * xMax;
                        const double az = dimnum == 3 ? a0z : 1.0;
                        par.wfc[g] = std::exp(-(std::pow(rad / (Rxy * a0x * 0.5), 2) +
                                                std::pow(par.z[k] / (Rxy * az * 0.5), 2)));
                        sum += std::abs(par.wfc[g]);
                        continue;
                    }
                    const double phi = -std::fmod(winding * std::atan2(par.y[j], par.x[i]), 2 * kPI);
                    const double e = std::exp(-(par.x[i] * par.x[i] / (Rxy * Rxy * a0x * a0x) +
                                                par.y[j] * par.y[j] / (Rxy * Rxy * a0y * a0y) +
                                                par.z[k] * par.z[k] / (Rxy * Rxy * a0z * a0z)));
                    par.wfc[g] = std::complex<double>(e * std::cos(phi), -e * std::sin(phi));
                    sum += std::abs(par.wfc[g]);
                }
        sum = std::sqrt(sum * dx * dy * dz);
        for (auto& v : par.wfc) v /= sum;
    } else if (par.wfc.size() != gSize) {
        throw std::runtime_error("the wavefunction read has the wrong size");
    }
}

gpue_params params_from_grid(const Grid& par) {
    gpue_params p;
    gpue_default_params(&p);
    p.dimnum = par.ival("dimnum");
    p.xDim = par.ival("xDim");
    p.yDim = par.ival("yDim");
    p.zDim = par.ival("zDim");
    p.xMax = par.dval("xMax");
    p.yMax = par.dval("yMax");
    p.zMax = par.dval("zMax");
    p.hbar = kHBAR;
    p.mass = par.dval("mass");
    p.omegaX = par.dval("omegaX");
    p.omegaY = par.dval("omegaY");
    p.omegaZ = par.dval("omegaZ");
    p.gammaY = par.dval("gammaY");
    p.x0_shift = par.dval("x0_shift");
    p.y0_shift = par.dval("y0_shift");
    p.z0_shift = par.dval("z0_shift");
    p.omega = par.dval("omega");
    p.interaction = par.dval("interaction");
    p.gDenConst = par.dval("gDenConst");
    p.gdt = par.dval("gdt");
    p.dt = par.dval("dt");
    p.gpe = par.bval("gpe") ? 1 : 0;
    p.corotating = par.bval("corotating") ? 1 : 0;
    p.gauge = par.Afn == "constant" ? GPUE_GAUGE_CONSTANT : GPUE_GAUGE_ROTATION;
    p.ramp = par.bval("ramp") ? 1 : 0;
    p.ramp_type = par.ival("ramp_type");
    p.precision = par.ival("precision");
    p.device = par.ival("device");
    return p;
}

void set_variables(Grid& par, int ev_type) {
    gpue_ctx* c = ensure_ctx(par);
    check(gpue_set_operators(c, ev_type), c, "set_variables");
}

double energy_calc(Grid& par) {
    gpue_ctx* c = ensure_ctx(par);
    check(gpue_set_wfc(c, par.wfc.data(), GPUE_MEM_HOST, GPUE_C128), c, "gpue_set_wfc");
    double E = 0;
    check(gpue_energy(c, &E), c, "energy_calc");
    return E;
}

// --------------------------------------------------------------- evolve --

// Tracker::findVortex on the resident state with radius mask_2d; prints the
// count as evolve() does and, when writing, the marks as vort_mark_<step>:
// one line "row,column,marker,winding" per marked plaquette (row = y index,
// column = x index, the marker index row*xDim + column), in findVortex's
// visiting order.
static void find_vortices(Grid& par, gpue_ctx* c, int step, bool write_it) {
    const double radius = par.dval("mask_2d");
    int32_t found = 0;
    check(gpue_find_vortices(c, radius, nullptr, GPUE_MEM_HOST, nullptr, 0, &found), c,
          "findVortex");
    std::printf("Located %d vortices\n", found);
    if (!write_it) return;
    std::vector<gpue_vortex> v((size_t)found);
    if (found > 0)
        check(gpue_find_vortices(c, radius, nullptr, GPUE_MEM_HOST, v.data(), found, &found),
              c, "findVortex");
    std::ofstream out(par.sval("data_dir") + "vort_mark_" + std::to_string(step));
    out << "#ROW,COLUMN,MARKER,WINDING\n";
    for (const gpue_vortex& m : v)
        out << m.i << ',' << m.j << ',' << m.marker << ',' << m.winding << '\n';
}


std::pair<int, int> resume_snapshot(Grid& par) {
    gpue_ctx* c = ensure_ctx(par);
    const std::string path = filecheck(par.sval("data_dir") + "snapshot.bin");
    int32_t g = 0;
    int64_t step = 0;
    check(gpue_snapshot_load(c, path.c_str(), &g, &step), c, "resume");
    std::printf("Resuming %s-time evolution at step %lld\n", g == 0 ? "imaginary" : "real",
                (long long)step);
    return {g, (int)step};
}

int evolve(Grid& par, int numSteps, unsigned gstate, const std::string& /*buffer*/) {
    gpue_ctx* c = ensure_ctx(par);
    const int start = par.ival("start_step");
    par.store("start_step", 0);  // applies to this call only
    if (start == 0)
        check(gpue_set_wfc(c, par.wfc.data(), GPUE_MEM_HOST, GPUE_C128), c, "gpue_set_wfc");
    const int ckpt = par.ival("checkpoint_every");
    const std::string data_dir = par.sval("data_dir");
    const int p = par.ival("printSteps");
    const bool write_it = par.bval("write_it");
    const bool ecalc = par.bval("energy_calc");
    const int every = ecalc ? (par.ival("energy_calc_steps") ? par.ival("energy_calc_steps") : p)
                            : 0;
    const bool ramp = par.bval("ramp");
    // src/evolution.cu:444-712
    const char* names[4] = {"wfc_0_const", "wfc_0_ramp", "wfc_ev", "wfc_ev_ramp"};
    const std::string fname = data_dir + names[(ramp ? 1 : 0) | (gstate << 1)];
    const std::string efile = data_dir + (gstate == 1 ? "energy.dat" : "energyi.dat");

    gpue_evolve_opts o;
    std::memset(&o, 0, sizeof o);
    o.energy_calc_steps = every;
    o.energy_calc_threshold = par.dval("energy_calc_threshold");
    o.norm_guard = -1;
    // 2D real time: findVortex at every print step (src/evolution.cu:483-486),
    // on the device; the later lattice analysis (vortPos/lsFit and the
    // optical lattice, src/evolution.cu:487-703) is not part of this build
    const bool track = gstate == 1 && par.ival("dimnum") == 2 && p > 0;
    int i = start;
    bool stopped = false;
    while (i < numSteps && !stopped) {
        if (ckpt > 0 && i > start && i % ckpt == 0)
            check(gpue_snapshot_save(c, (data_dir + "snapshot.bin").c_str(), (int32_t)gstate, i),
                  c, "snapshot");
        if (write_it && p > 0 && i % p == 0) {  // the state after i steps
            check(gpue_get_wfc(c, par.wfc.data(), GPUE_MEM_HOST, GPUE_C128), c, "gpue_get_wfc");
            fileio::write_out(fname, par.wfc, i);
        }
        if (track && i % p == 0) find_vortices(par, c, i, write_it);
        // one call up to the next print point or just past the next check
        int next = numSteps;
        if ((write_it || track) && p > 0) next = std::min(next, (i / p + 1) * p);
        if (ckpt > 0) next = std::min(next, (i / ckpt + 1) * ckpt);
        int check_step = -1;
        if (every > 0) {
            const int nc = ((i + every - 1) / every) * every;
            if (nc < numSteps && nc + 1 <= next) {
                next = nc + 1;
                check_step = nc;
            }
        }
        o.step_offset = i;
        gpue_evolve_result r;
        check(gpue_evolve(c, next - i, (int32_t)gstate, &o, &r), c, "evolve");
        if (r.n_energies > 0) {
            std::ofstream eo(efile, check_step == 0 ? std::ios::out : std::ios::app);
            eo << r.energy << '\n';
            par.store("energy", r.energy);
            std::printf("Energy[t@%d]=%E\n", check_step, r.energy);
        }
        i += r.steps_done;
        if (r.early_stop) {
            std::printf("Stopping early at step %d with energy %E\n", i - 1, r.energy);
            stopped = true;
        }
    }
    check(gpue_get_wfc(c, par.wfc.data(), GPUE_MEM_HOST, GPUE_C128), c, "gpue_get_wfc");
    return i;
}

// --------------------------------------------------------------- fileio --

namespace fileio {

std::vector<std::complex<double>> read_in(const std::string& fileR, const std::string& fileI,
                                          size_t n) {
    std::vector<std::complex<double>> v(n);
    for (int part = 0; part < 2; ++part) {
        FILE* f = std::fopen((part ? fileI : fileR).c_str(), "r");
        if (!f) throw std::runtime_error("cannot read " + (part ? fileI : fileR));
        size_t i = 0;
        double d;
        while (i < n && std::fscanf(f, "%lE", &d) == 1) {
            if (part) v[i].imag(d);
            else v[i].real(d);
            ++i;
        }
        std::fclose(f);
        if (i != n) throw std::runtime_error("too few values in " + (part ? fileI : fileR));
    }
    return v;
}

void write_out(const std::string& file, const std::vector<std::complex<double>>& data,
               int step) {
    for (int part = 0; part < 2; ++part) {
        const std::string name = file + (part ? "i_" : "_") + std::to_string(step);
        FILE* f = std::fopen(name.c_str(), "w");
        if (!f) throw std::runtime_error("cannot write " + name);
        for (const auto& v : data) std::fprintf(f, "%.16e\n", part ? v.imag() : v.real());
        std::fclose(f);
    }
}

void write_out_double(const std::string& file, const std::vector<double>& data, int step) {
    const std::string name = file + "_" + std::to_string(step);
    FILE* f = std::fopen(name.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + name);
    for (double v : data) std::fprintf(f, "%.16e\n", v);
    std::fclose(f);
}

}  // namespace fileio

}  // namespace gpue_host
