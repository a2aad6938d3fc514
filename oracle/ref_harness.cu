// ref_harness.cu -- TEST INFRASTRUCTURE ONLY.
//
// Drives GPUE's own CUDA build (its parseArgs, init, set_variables, evolve and
// energy_calc, compiled unmodified from the reference sources) on a seeded
// initial wavefunction, and writes the final device wavefunction and energy
// in binary/text so the tests can pin the CPU oracle and the CUDA product to
// the reference itself.
//
// GPUE works in SI units with hbar = 1.05457148e-34 (include/constants.h:20)
// and forces the Rb-87 mass (src/init.cu:98).  The dimensionless problem
// (hbar = m = 1) maps onto it exactly with a time unit of 1 s and a length
// unit L = sqrt(hbar/m):  x_SI = x L,  p_SI = p / L,  t and omega unchanged,
// E_SI = hbar E,  psi_SI = psi / L^(d/2),  gN_SI = g hbar L^d.  The gauge
// field A = omega*(-y wx, x wy) and the +m|A|^2/2 term in V map the same way.
//
// Usage (key=value):
//   gpue_ref_harness dim=2 n=64 box=10 wx=1 wy=1 wz=1 gamma=1 g=100 gpe=1
//       omega=0 gauge=0 gdt=1e-4 dt=1e-4 gsteps=100 esteps=0 energy_every=0
//       [ramp=1 ramp_type=1]
//       psi0=in.bin out=prefix data=/tmp/dir
// Writes prefix_imag.bin / prefix_real.bin (complex128, x fastest, hbar=m=1
// units) and prefix_imag.txt / prefix_real.txt ("energy <E>" and
// "last_check_energy <E>", plus "evolve_s <seconds>" of the evolve() call).
//
//   gpue_ref_harness mode=vortex n=128 box=8 radius=5 psi0=in.bin out=prefix
// runs only GPUE's host-side Tracker::findVortex (src/tracker.cu:102-166) on
// the n x n complex128 state in psi0 with GPUE's x grid, and writes the marker
// array (int32, n*n) to prefix_vortex.bin and "found <count>" to
// prefix_vortex.txt.  This mode makes no CUDA call and needs no GPU.
//
//   gpue_ref_harness mode=ast doubles=names.txt exprs=exprs.txt out=prefix
//   gpue_ref_harness mode=ast doubles=names.txt param=file.cfg out=prefix
// runs only GPUE's host-side equation parser (parse_eqn, find_element_num and
// tree_to_array, src/dynamic.cu:227-530) with a Grid holding the doubles of
// names.txt ("name value" lines).  With exprs, every line is one expression
// parsed as entry "V"; with param, the file is read line by line as
// parse_param_file does (src/dynamic.cu:187-222: spaces dropped, lines without
// '=' continue the previous entry, V gets +0.5*mass*(Ax*Ax+Ay*Ay+Az*Az) unless
// it is the last entry) and each entry goes through allocate_eqn's host part
// (src/dynamic.cu:162-185; the device copy is left out).  prefix_ast.txt gets,
// per entry, "entry <name> <count> <time_flag>" and then one line per
// EqnNode_gpu: "<val as %a> <is_dynamic> <var> <left> <right> <op_num>", with
// op_num written as 0 for leaves (GPUE leaves it unset there).  No CUDA call.

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "constants.h"
#include "ds.h"
#include "dynamic.h"
#include "evolution.h"
#include "init.h"
#include "parser.h"
#include "split_op.h"
#include "tracker.h"

namespace {

std::map<std::string, std::string> g_kv;

std::string get(const char* k, const char* def) {
    auto it = g_kv.find(k);
    return it == g_kv.end() ? std::string(def) : it->second;
}
double getd(const char* k, double def) {
    auto it = g_kv.find(k);
    return it == g_kv.end() ? def : atof(it->second.c_str());
}
int geti(const char* k, int def) {
    auto it = g_kv.find(k);
    return it == g_kv.end() ? def : atoi(it->second.c_str());
}
std::string fmt(double v) {
    char b[64];
    snprintf(b, sizeof b, "%.17g", v);
    return b;
}

void dump(Grid& par, const std::string& path, int gsize, double L, int dim, double secs) {
    double2* dev = par.cufftDoubleComplexval("wfc_gpu");
    std::vector<double2> h(gsize);
    cudaMemcpy(h.data(), dev, sizeof(double2) * gsize, cudaMemcpyDeviceToHost);
    double s = std::pow(L, 0.5 * dim);
    for (auto& v : h) { v.x *= s; v.y *= s; }
    FILE* f = fopen((path + ".bin").c_str(), "wb");
    fwrite(h.data(), sizeof(double2), gsize, f);
    fclose(f);
    double e = energy_calc(par, dev) / HBAR;
    double last = par.dval("energy") / HBAR;
    FILE* t = fopen((path + ".txt").c_str(), "w");
    fprintf(t, "energy %.17g\nlast_check_energy %.17g\nevolve_s %.6f\n", e, last, secs);
    fclose(t);
}

void ast_entry(Grid& par, FILE* out, const std::string& name, const std::string& expr) {
    par.store(name + "_time", false);
    EqnNode tree = parse_eqn(par, expr, name);
    int num = 0;
    find_element_num(tree, num);
    std::vector<EqnNode_gpu> arr(num);
    int count = 0;
    tree_to_array(tree, arr.data(), count);
    par.store(name, tree);
    fprintf(out, "entry %s %d %d\n", name.c_str(), num, par.bval(name + "_time") ? 1 : 0);
    for (const EqnNode_gpu& e : arr)
        fprintf(out, "%a %d %d %d %d %d\n", e.val, e.is_dynamic ? 1 : 0, (int)e.var, e.left,
                e.right, e.left >= 0 ? e.op_num : 0);
}

int ast_mode() {
    Grid par;
    {
        FILE* f = fopen(get("doubles", "doubles.txt").c_str(), "r");
        if (!f) {
            fprintf(stderr, "cannot read doubles\n");
            return 2;
        }
        char name[256];
        double v;
        while (fscanf(f, "%255s %lf", name, &v) == 2) par.store(std::string(name), v);
        fclose(f);
    }
    FILE* out = fopen((get("out", "ref") + "_ast.txt").c_str(), "w");
    const std::string param = get("param", "");
    if (!param.empty()) {
        std::ifstream file(param);
        std::string line, val_string, eqn_string;
        while (std::getline(file, line)) {
            line.erase(std::remove_if(line.begin(), line.end(), ::isspace), line.end());
            const size_t it = line.find('=');
            if (it == std::string::npos) {
                eqn_string += line;
            } else {
                if (!val_string.empty()) {
                    if (val_string == "V") eqn_string += "+0.5*mass*(Ax*Ax+Ay*Ay+Az*Az)";
                    ast_entry(par, out, val_string, eqn_string);
                    val_string.clear();
                    eqn_string.clear();
                }
                val_string = line.substr(0, it);
                eqn_string = line.substr(it + 1);
            }
        }
        ast_entry(par, out, val_string, eqn_string);
    } else {
        std::ifstream file(get("exprs", "exprs.txt"));
        std::string line;
        while (std::getline(file, line))
            if (!line.empty()) ast_entry(par, out, "V", line);
    }
    fclose(out);
    return 0;
}

int vortex_mode() {
    const int n = geti("n", 64);
    const double xMax = getd("box", 10);
    std::vector<double2> wfc((size_t)n * n);
    FILE* f = fopen(get("psi0", "psi0.bin").c_str(), "rb");
    if (!f || fread(wfc.data(), sizeof(double2), wfc.size(), f) != wfc.size()) {
        fprintf(stderr, "cannot read psi0\n");
        return 2;
    }
    fclose(f);
    // generate_p_space's x (src/operators.cu:336-343)
    std::vector<double> x(n);
    const double dx = xMax / (n >> 1);
    for (int i = 0; i < n / 2; ++i) {
        x[i] = -xMax + i * dx;
        x[i + n / 2] = i * dx;
    }
    std::vector<int> marker((size_t)n * n, 0);
    const int found = Tracker::findVortex(marker.data(), wfc.data(), getd("radius", 1.0), n,
                                          x.data(), 0);
    const std::string out = get("out", "ref");
    FILE* b = fopen((out + "_vortex.bin").c_str(), "wb");
    fwrite(marker.data(), sizeof(int), marker.size(), b);
    fclose(b);
    FILE* t = fopen((out + "_vortex.txt").c_str(), "w");
    fprintf(t, "found %d\n", found);
    fclose(t);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        size_t eq = a.find('=');
        if (eq != std::string::npos) g_kv[a.substr(0, eq)] = a.substr(eq + 1);
    }
    if (get("mode", "") == "vortex") return vortex_mode();
    if (get("mode", "") == "ast") return ast_mode();
    const int dim = geti("dim", 2);
    const int n = geti("n", 64);
    const int gsteps = geti("gsteps", 0), esteps = geti("esteps", 0);
    const double mass = 1.4431607e-25;  // the mass init() stores
    const double L = std::sqrt(HBAR / mass);
    const std::string data = get("data", "/tmp/gpue_ref_data");

    std::vector<std::string> a = {"gpue", "-c", std::to_string(dim),
                                  "-x", std::to_string(n), "-y", std::to_string(n)};
    if (dim == 3) { a.push_back("-z"); a.push_back(std::to_string(n)); }
    // -c 3 resets box_size, so -b comes after it
    for (auto s : {std::string("-b"), fmt(getd("box", 10) * L),
                   std::string("-X"), fmt(getd("wx", 1)), std::string("-Y"), fmt(getd("wy", 1)),
                   std::string("-Z"), fmt(getd("wz", 1)), std::string("-G"), fmt(getd("gamma", 1)),
                   std::string("-T"), fmt(getd("gdt", 1e-4)), std::string("-t"), fmt(getd("dt", 1e-4)),
                   std::string("-g"), std::to_string(gsteps), std::string("-e"), std::to_string(esteps),
                   std::string("-p"), std::to_string((gsteps > esteps ? gsteps : esteps) + 1),
                   std::string("-f"), std::string("-d"), data})
        a.push_back(s);
    if (geti("gpe", 1)) a.push_back("-s");
    if (geti("gauge", 0)) {
        a.push_back("-l");
        a.push_back("-w");
        a.push_back(fmt(getd("omega", 0)));
    }
    if (geti("ramp", 0)) {  // parseArgs' -R <ramp_type> (src/parser.cu:188-194)
        a.push_back("-R");
        a.push_back(std::to_string(geti("ramp_type", 1)));
    }
    std::vector<char*> av;
    for (auto& s : a) av.push_back(const_cast<char*>(s.c_str()));
    av.push_back(nullptr);
    Grid par = parseArgs((int)a.size(), av.data());

    int gsize = n * n * (dim == 3 ? n : 1);
    double2* wfc = (double2*)malloc(sizeof(double2) * gsize);
    {
        FILE* f = fopen(get("psi0", "psi0.bin").c_str(), "rb");
        if (!f || fread(wfc, sizeof(double2), gsize, f) != (size_t)gsize) {
            fprintf(stderr, "cannot read psi0\n");
            return 2;
        }
        fclose(f);
        double s = std::pow(L, -0.5 * dim);
        for (int i = 0; i < gsize; ++i) { wfc[i].x *= s; wfc[i].y *= s; }
    }
    par.store("read_wfc", true);
    par.store("wfc", wfc);
    int every = geti("energy_every", 0);
    par.store("energy_calc", true);
    par.store("energy_calc_steps", every > 0 ? every : 1 << 30);
    par.store("energy_calc_threshold", getd("threshold", -1.0));
    par.store("energy", 0.0);

    init(par);
    double gN = getd("g", 0) * HBAR * std::pow(L, dim);
    par.store("interaction", gN / par.dval("gDenConst"));

    std::string buf;
    std::string out = get("out", "ref");
    if (gsteps > 0) {
        set_variables(par, 0);
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        evolve(par, gsteps, 0, buf);
        cudaDeviceSynchronize();
        double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        dump(par, out + "_imag", gsize, L, dim, s);
    }
    if (esteps > 0) {
        set_variables(par, 1);
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        evolve(par, esteps, 1, buf);
        cudaDeviceSynchronize();
        double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        dump(par, out + "_real", gsize, L, dim, s);
    }
    return 0;
}
