// host.h -- the C++ host layer over the C ABI: GPUE's command line, init(),
// file formats and an evolve(Grid&, ...) that runs the step on the library.
//
// A GPUE user keeps the same flags and files; the step itself runs through
// gpue_evolve on a context the Grid owns.
#pragma once

#include <string>
#include <utility>

#include "grid.h"

namespace gpue_host {

// GPUE's parseArgs (src/parser.cu:7-471): defaults, then the flags.  Flags
// of analyses outside the step (vortex tracking, kicks, graphs) are stored
// like GPUE stores them and otherwise unused.  Three long options are read
// before the getopt flags: --precision=fp64|fp32, --autotune, --print-params.
Grid parse_args(int argc, char** argv);

// GPUE's init() (src/init.cu:40-356) for what the step needs: Rb-87 units,
// derived lengths and steps, the coordinate axes and -- unless a wavefunction
// was read -- the standard initial state (kstd_wfc, src/operators.cu:1031-
// 1050) normalised as GPUE does it.  Throws std::runtime_error on options
// this build does not implement.
void init(Grid& par);

// The gpue_params the Grid's keys describe (src/evolution.cu:266-332).
gpue_params params_from_grid(const Grid& par);

// set_variables(par, ev_type) (src/init.cu:358-497).
void set_variables(Grid& par, int ev_type);

// evolve(par, numSteps, gstate, buffer) (include/evolution.h:54-57): the
// steps run on the device; par.wfc is read first and holds the final state
// after.  With write_it, the state after every printSteps-th step is written
// as GPUE names it (wfc_0_const_<i>, wfc_ev_<i>, ...); with energy_calc, the
// check energies are appended to energyi.dat / energy.dat and "energy" holds
// the last one.  Returns the steps run.
// With checkpoint_every = K > 0 a binary snapshot (gpue_snapshot_save) of
// the state after every K-th step goes to <data_dir>snapshot.bin; with
// "start_step" = s > 0 the loop starts at step s on the state the context
// already holds (a resumed run) instead of reading par.wfc.
int evolve(Grid& par, int numSteps, unsigned gstate, const std::string& buffer);

// --resume: loads <data_dir>snapshot.bin into the context; returns its phase
// (0 imaginary, 1 real) and step.
std::pair<int, int> resume_snapshot(Grid& par);

// energy_calc(par, wfc) (src/split_op.cu:208-375) of the current state.
double energy_calc(Grid& par);

// GPUE's text formats (src/fileIO.cu:13-72): one "%.16e" value per line,
// real parts in <file>_<step>, imaginary parts in <file>i_<step>.
namespace fileio {
std::vector<std::complex<double>> read_in(const std::string& fileR, const std::string& fileI,
                                          size_t n);
void write_out(const std::string& file, const std::vector<std::complex<double>>& data,
               int step);
void write_out_double(const std::string& file, const std::vector<double>& data, int step);
}  // namespace fileio

}  // namespace gpue_host
