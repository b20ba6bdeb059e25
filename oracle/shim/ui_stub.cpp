// The oracle runs BOSampleStepper with an empty iter_cmd, so the command
// interpreter (src/UserInterface.cpp, excluded from this build) is never
// entered.  This definition only satisfies the linker for the call that
// src/BOSampleStepper.cpp:474-486 guards with `if ( !iter_cmd_.empty() )`.
// Test infrastructure, not product.
#include <cstdio>
#include <cstdlib>
#include "UserInterface.h"
void UserInterface::processCmds(std::istream&, const std::string, bool)
{ std::fprintf(stderr, "iter_cmd not supported\n"); std::abort(); }
