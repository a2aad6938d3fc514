// main.cpp -- the gpue command line: GPUE's main() (src/init.cu:500-568)
// over the B200 step.  Same flags and files as GPUE; five extra options:
//   --precision=fp32   the fused complex64 form (default fp64, the replica)
//   --autotune         time the FFT plans for this grid before stepping
//   --print-params     print the parameters the step would use and exit
//   --checkpoint-every=K  binary snapshot of the state every K steps
//                      (<data_dir>snapshot.bin, replaced each time)
//   --resume           continue from <data_dir>snapshot.bin
#include <chrono>
#include <cstdio>
#include <iostream>

#include "host.h"

using namespace gpue_host;

int main(int argc, char** argv) {
    try {
        Grid par = parse_args(argc, argv);
        const int gSize = par.ival("xDim") * par.ival("yDim") * par.ival("zDim");
        if (par.bval("read_wfc"))
            par.wfc = fileio::read_in(par.sval("infile"), par.sval("infilei"), (size_t)gSize);
        init(par);
        if (par.bval("print_params")) {
            const gpue_params p = params_from_grid(par);
            std::printf("dimnum=%d\nxDim=%d\nyDim=%d\nzDim=%d\n", p.dimnum, p.xDim, p.yDim,
                        p.zDim);
            std::printf("xMax=%.17g\nyMax=%.17g\nzMax=%.17g\n", p.xMax, p.yMax, p.zMax);
            std::printf("hbar=%.17g\nmass=%.17g\n", p.hbar, p.mass);
            std::printf("omegaX=%.17g\nomegaY=%.17g\nomegaZ=%.17g\ngammaY=%.17g\n", p.omegaX,
                        p.omegaY, p.omegaZ, p.gammaY);
            std::printf("omega=%.17g\ninteraction=%.17g\ngDenConst=%.17g\n", p.omega,
                        p.interaction, p.gDenConst);
            std::printf("gdt=%.17g\ndt=%.17g\ngpe=%d\ncorotating=%d\ngauge=%d\n", p.gdt, p.dt,
                        p.gpe, p.corotating, p.gauge);
            std::printf("ramp=%d\nramp_type=%d\nprecision=%d\n", p.ramp, p.ramp_type,
                        p.precision);
            std::printf("gsteps=%d\nesteps=%d\n", par.ival("gsteps"), par.ival("esteps"));
            for (const char* k : {"x0_shift", "y0_shift", "z0_shift", "fudge", "Rxy", "a0x",
                                  "a0y", "a0z", "dx", "dy", "dz"})
                std::printf("%s=%.17g\n", k, par.dval(k));
            std::printf("energy_calc_steps=%d\nenergy_calc_threshold=%.17g\n",
                        par.bval("energy_calc") ? par.ival("energy_calc_steps") : -1,
                        par.dval("energy_calc_threshold"));
            return 0;
        }
        const auto t0 = std::chrono::steady_clock::now();
        const std::string data_dir = par.sval("data_dir");
        const std::string buffer;
        if (par.bval("write_file")) {
            par.write(data_dir + "Params.dat");
            fileio::write_out(data_dir + "WFC", par.wfc, 0);
            fileio::write_out_double(data_dir + "x", par.x, 0);
            fileio::write_out_double(data_dir + "y", par.y, 0);
            fileio::write_out_double(data_dir + "z", par.z, 0);
        }
        // --resume: continue from <data_dir>snapshot.bin (its phase and step)
        int phase = 0;
        if (par.bval("resume")) {
            const auto r = resume_snapshot(par);
            phase = r.first;
            par.store("start_step", r.second);
        }
        if (phase == 0 && par.ival("gsteps") > 0) {
            std::cout << "Imaginary-time evolution started..." << '\n';
            set_variables(par, 0);
            evolve(par, par.ival("gsteps"), 0, buffer);
            if (par.bval("write_file")) fileio::write_out(data_dir + "wfc_0_final", par.wfc, 0);
        }
        if (par.ival("esteps") > 0) {
            std::cout << "real-time evolution started..." << '\n';
            set_variables(par, 1);
            evolve(par, par.ival("esteps"), 1, buffer);
            if (par.bval("write_file")) fileio::write_out(data_dir + "wfc_ev_final", par.wfc, 0);
        }
        const double s =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::cout << "done evolving" << '\n' << "Total time: " << s << " seconds\n";
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "gpue: %s\n", e.what());
        return 1;
    }
}
