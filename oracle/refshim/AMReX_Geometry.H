/* shim: forwards to vd_amrex_shim.H (test infrastructure only) */
#include "vd_amrex_shim.H"
