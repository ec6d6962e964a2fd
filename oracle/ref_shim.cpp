// ref_shim.cpp - replaces QPandaSDK/QuantumInstructionHandle/QuantumGates.cpp
// when the reference CPU backend is compiled from its own sources into
// oracle/_ref/ (see oracle/Makefile).  TEST INFRASTRUCTURE ONLY.
//
// The reference file holds the QuantumGates ctor/dtor and randGenerator(), a
// Park-Miller 16807 generator seeded once from the wall clock
// (QuantumGates.cpp:46-85).  Here the seed is explicit and a caller can inject
// the next value, so that measurements use known uniforms.  The generator
// never returns 0, so "randGenerator() > error_rate(=0)" still applies every
// gate.
#include "QuantumGates.h"

static int g_seed = 20180501;
static bool g_have_next = false;
static double g_next = 0.0;

QuantumGates::QuantumGates() {}
QuantumGates::~QuantumGates() {}

double QuantumGates::randGenerator()
{
    if (g_have_next) {
        g_have_next = false;
        return g_next;
    }
    const int ia = 16807, im = 2147483647, iq = 127773, ir = 2836;
    int x = ia * (g_seed % iq) - ir * (g_seed / iq);
    if (x < 0) x += im;
    g_seed = x;
    return (double)x / im;
}

extern "C" void ref_rng_seed(int seed) { g_seed = seed ? seed : 1; g_have_next = false; }
extern "C" void ref_rng_set_next(double u) { g_next = u; g_have_next = true; }
