// The oracle never sets an external potential (Sample::vext stays null), so
// the Xerces-dependent src/ExternalPotential.cpp is not compiled.  These
// definitions only satisfy the linker for the calls that
// src/EnergyFunctional.cpp:88,364-369 guards with `if ( s_.vext )`.
// Test infrastructure, not product.
#include <cstdio>
#include <cstdlib>
#include "ExternalPotential.h"
void ExternalPotential::update(const ChargeDensity&)
{ std::fprintf(stderr, "external potential not supported\n"); std::abort(); }
double ExternalPotential::compute_eext(const ChargeDensity&)
{ std::fprintf(stderr, "external potential not supported\n"); std::abort(); return 0; }
