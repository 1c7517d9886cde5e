// run_rewl_b200.hpp — the B200 engine behind the reference sampler's own run_rewl signature.
//
// The reference's seam for the sampling path is
//
//     RewlResult run_rewl(const ParallelContext&, std::shared_ptr<const Couplings>,
//                         const RunConfig&);                     (include/wl/parallel.hpp:35-36)
//
// run_rewl_b200 takes the same arguments and returns the same RewlResult, computed by the
// engine in libwlg.so through its C-ABI (include/wlg.h).  It is compiled against the
// reference's headers, so a program that calls wl::run_rewl switches to the GPU by calling
// wl::run_rewl_b200 instead (apps/wl_run.cpp:126 and :176 are the two call sites of wl_run;
// wl_run_b200.hpp retargets both without editing the file).
//
// What it does beyond the call:
//   - the couplings are exported through the public Couplings interface (size(), at(i, j),
//     backend_name(); include/wl/physics.hpp:41-49): the dense backend as its n x n matrix,
//     the CSR backend as the rows of its non-zero couplings.  For CSR that is n^2 calls of
//     at(), each a scan of one row (the same cost as one reference local_fields call), spread
//     over the OpenMP threads;
//   - one process drives one GPU: a ParallelContext of more than one rank is rejected;
//   - errors come back as the reference's exception types with the engine's messages, which
//     repeat the reference's (std::invalid_argument, std::runtime_error, std::logic_error,
//     std::out_of_range).
#pragma once

#include <memory>

#include "wl/parallel.hpp"

namespace wl {

[[nodiscard]] RewlResult run_rewl_b200(const ParallelContext& context, std::shared_ptr<const Couplings> couplings,
                                       const RunConfig& config);

}  // namespace wl
