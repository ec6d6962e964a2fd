// qrunes_runner.cpp - TEST HARNESS: QRunes programs end to end through the
// reference's own parser (QRunesParser/) and dispatcher
// (QuantumInstructionHandle/QuantumInstructionGet.cpp, Instruction.cpp),
// compiled from the reference sources, with either the reference CPU backend
// (CPUQuantumGates.cpp) or the B200 backend (qpanda_b200/host/B200QuantumGates)
// behind the QuantumGates interface.  The QuantumGates base (constructor and
// the 16807 generator) comes from oracle/ref_shim.cpp, seeded explicitly.
//
// Backend 3 is the reference's own GPU compute unit (GPUQuantumGates.cpp,
// unmodified), which dlopens "libGPUEmulator.so" - here this repository's
// qpanda_b200/_lib/libGPUEmulator.so, loaded by the caller beforehand - and is
// handed the same generator as the other backends.
//
// qr_run mirrors QPandaSDK::loadFile + QPandaSDK::run (QPandaAPI.cpp:59-96,
// 131-211): parse, initState, then per shot transmit() - an END node (reset
// to |0...0>, QuantumInstructionHandleAPI.cpp:96-100) followed by every node -
// and count the classical registers (countState, :264-285); a program with
// PMEASURE runs once and reports the top-10 outcomes as bitstrings.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>
#include <string>

#include <dlfcn.h>

#include "CPUQuantumGates.h"
#include "GPUQuantumGates.h"
#include "QRunesParserAPI.h"
#include "QuantumInstructionGet.h"
#include "B200QuantumGates.h"

extern "C" void ref_rng_seed(int seed);

// The GPU compute unit's gates draw from the program's QuantumGates generator.
static QuantumGates *g_rng_owner = nullptr;
static double program_rng() { return g_rng_owner->randGenerator(); }

static bool transmit(QList &list, QuantumGateParam *param, QuantumGates *g)
{
    QuantumInstructionGet *get = QuantumInstructionGet::getInstance();
    QNode endProg = {END, nullptr};
    if (!get->transmit(&endProg, param, g)) return false;
    for (QNode *p = list.qList.head->next; p; p = p->next)
        if (!get->transmit(p, param, g)) return false;
    return true;
}

static std::string to_binary(size_t v, size_t len)
{
    std::string s;
    for (size_t i = 0; i < len; ++i) s += ((v >> (len - 1 - i)) & 1) ? '1' : '0';
    return s;
}

// backend: 0 = reference CPU, 1 = B200 complex128, 2 = B200 complex64,
// 3 = the reference's GPUQuantumGates over libGPUEmulator.so.
// Writes "MEASURE bits:freq,..." or "PMEASURE bits:prob,..." into out.
// Returns the qubit count, or a negative value on failure.
extern "C" int qr_run(const char *path, int backend, int seed, int repeat, char *out, size_t out_len)
{
    std::string file(path);
    QList list;
    int n = QRunesParser(file, list);
    if (n <= 0 || n > 30) return -1;
    std::unique_ptr<QuantumGates> g;
    if (backend == 0) {
        g.reset(new CPUQuantumGates());
    } else if (backend == 3) {
        void *emu = dlopen("libGPUEmulator.so", RTLD_NOW | RTLD_NOLOAD);
        if (!emu) return -5;
        typedef void (*set_rng_fn)(double (*)(void));
        set_rng_fn set_rng = reinterpret_cast<set_rng_fn>(dlsym(emu, "qs_gpuemu_set_rng"));
        if (!set_rng) return -5;
        try {
            g.reset(new GPUQuantumGates());
        } catch (...) {
            return -5;
        }
        g_rng_owner = g.get();
        set_rng(&program_rng);
    } else {
        g.reset(new B200QuantumGates(backend == 2 ? QS_C64 : QS_C128));
    }
    QuantumGateParam param;
    param.mQuantumBitNumber = n;
    if (g->initState(&param) != qErrorNone) return -2;
    ref_rng_seed(seed);
    std::map<std::string, double> res;
    std::string kind;
    if (!transmit(list, &param, g.get())) return -3;
    if (param.mPMeasureSize == 0) {
        kind = "MEASURE";
        for (int shot = 0; shot < repeat; ++shot) {
            if (shot && !transmit(list, &param, g.get())) return -3;
            std::stringstream ss;
            for (auto &kv : param.mReturnValue) ss << kv.second;
            std::string b = ss.str();
            std::reverse(b.begin(), b.end());
            res[b] += 1.0;
        }
        for (auto &kv : res) kv.second /= repeat;
    } else {
        kind = "PMEASURE";
        for (auto &kv : param.mPMeasure) res[to_binary(kv.first, param.mPMeasureSize)] = kv.second;
    }
    std::stringstream os;
    os.precision(17);
    os << kind;
    bool first = true;
    for (auto &kv : res) {
        os << (first ? " " : ",") << kv.first << ":" << kv.second;
        first = false;
    }
    std::string s = os.str();
    // the GPU compute unit's destructor does not free its state
    if (backend == 3) {
        g->destroyState((size_t)n);
        typedef void (*set_rng_fn)(double (*)(void));
        void *emu = dlopen("libGPUEmulator.so", RTLD_NOW | RTLD_NOLOAD);
        if (emu) reinterpret_cast<set_rng_fn>(dlsym(emu, "qs_gpuemu_set_rng"))(nullptr);
    }
    if (s.size() + 1 > out_len) return -4;
    memcpy(out, s.c_str(), s.size() + 1);
    return n;
}
