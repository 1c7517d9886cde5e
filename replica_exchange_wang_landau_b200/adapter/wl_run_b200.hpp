// wl_run_b200.hpp — force-included (g++ -include) when the reference's unmodified
// apps/wl_run.cpp is compiled into wl_run_b200: both of its run_rewl call sites (the
// adaptive-window pilots, apps/wl_run.cpp:126, and the production run, :176) then call
// run_rewl_b200, so the program keeps its INI/CLI, geometry loading, stitching and every
// output file and runs the sampling on the GPU.
//
// parallel.hpp is included (and its include guard set) before the macro, so its own
// declaration of run_rewl is untouched; the macro renames only the calls that follow.
#pragma once

#include "run_rewl_b200.hpp"

#define run_rewl run_rewl_b200
