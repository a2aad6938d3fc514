// batch_mega.cuh -- many independent solves of uneven grid sizes in one
// persistent launch.
//
// A segment of a batched run (the time steps up to the next energy check) is
// a list of pass instances: pass r of solve s, for every solve and every
// pass r of its pass list (its own schedule: 2D or 3D, gauge or not).  The
// instances are ordered by pass index (pass 0 of every solve, then pass 1, ...)
// and cut into work items of `chunk` consecutive tiles (about 32K points), the
// items numbered consecutively: a ticket, mapped to its instance by a table.
// One launch of resident CTAs walks the tickets with an atomic counter; before
// an item of pass r of solve s, the CTA waits until pass r-1 of that solve has
// finished all its items (a per-instance completion counter).  Tickets are taken in order and
// a tile only ever waits on tiles with smaller tickets, which CTAs that are
// already running took, so the walk always progresses whatever the number of
// resident CTAs; the wait is bounded all the same (a flag records a wait that
// gave up, and the run reports GPUE_ERR_TIMEOUT).
//
// Every tile runs the line-pass body of its solve's length and axis (the same
// code as the single-solve passes), with a fixed 256 threads per CTA: C =
// 256/P lines per tile for a plan of P threads per line.  A solve's tiling
// and reductions depend only on its own size, so its results are the same
// alone and in any mix.  Converged solves (active flag 0) have their tiles
// counted as done without work.
#pragma once

#include "pass.cuh"

namespace gpue {

constexpr int kMegaThreads = 256;

struct MegaPass {
    long start;   // first ticket (work item) of this instance
    int nitems;   // its work items
    int ntiles;
    int chunk;    // tiles per work item (the last may hold fewer)
    int dep;      // instance this one waits for (pass r-1 of the solve), -1 for none
    int kind;     // tile body: index into the compiled length list, x 2, + strided
    int args;     // index into MegaArgs::args
};

struct MegaArgs {
    const MegaPass* passes;
    const int* item_pass;    // [total]: the instance of each work item
    int npass;
    long total;              // tickets
    const PassArgs* args;
    unsigned long long* ticket;  // zero before the launch
    int* done;                   // [npass] finished items, zero before the launch
    int* err;                    // set when a dependency wait gave up
};

constexpr unsigned kMegaWaitPolls = 1u << 24;

}  // namespace gpue
