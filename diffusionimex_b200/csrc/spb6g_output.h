// Output formats of the reference's main(): the 17-column profile
// (write_profile, src/SPB6_PC_IMEX_omp.cpp:1083-1094), the pressure probe
// (probe_write, :1191-1197), snapshot names (snap_name, physics :973) and the
// end-of-run statistics line (:1425-1427).  Host code: the cell diagnostics are
// evaluated on the host in FP64 with the reference's formulas (cell_diag,
// physics :1161-1172; prim_of :893-902), so a state equal to the reference's
// prints the same text.
#pragma once
#include <cstdint>
#include <string>

#include "../../include/spb6g.h"

namespace spb6g {
namespace out {

// The 15 diagnostics of one cell (AoS record of 8 conservative values):
// p u v rho alpha2 Y2 rho1 rho2 c_frozen c_wood T1 T2 p1 p2 g1-g2.
void cell_diag(const spb6g_config& cf, const double* Q, double* o);
// The profile of every interior cell (state in the AoS layout of spb6g.h).
int write_profile(const spb6g_config& cf, const double* U, const char* path, int prec);
// One probe line "t p Y2 alpha2 T1" of the cell nearest (px, py); first: truncate the file.
int write_probe(const spb6g_config& cf, const double* U, double t, double px, double py, const std::string& path, bool first);
// <out>_s<k>.dat (a trailing ".dat" of out is replaced).
std::string snap_name(const std::string& out, size_t k);
// Sums of m1, m2 and E over the interior cells in the reference's loop order.
void conserved_totals(const spb6g_config& cf, const double* U, double M[3]);

}  // namespace out
}  // namespace spb6g
