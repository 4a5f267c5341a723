// Shim header (test infrastructure): see amrex_shim.H.
#pragma once
#include "amrex_shim.H"
