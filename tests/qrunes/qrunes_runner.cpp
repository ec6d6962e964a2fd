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
// qr_run_ex with `sample` set runs that loop the way a B200 integration of
// QPandaSDK::run would: a dry probe pass (B200QuantumGates::beginProbe)
// tells whether every MEASURE is terminal; if so the program runs once in
// deferred-measurement mode and the shots come from
// B200QuantumGates::sampleDeferred, with the same generator stream; else the
// per-shot loop runs as before.  *runs receives the number of simulations.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

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
extern "C" int qr_run_ex(const char *path, int backend, int seed, int repeat, int sample, char *out,
                         size_t out_len, int *runs)
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
    B200QuantumGates *b = (backend == 1 || backend == 2) ? static_cast<B200QuantumGates *>(g.get()) : nullptr;
    bool deferred = false;
    if (sample && b) {
        QuantumGateParam probe;
        probe.mQuantumBitNumber = n;
        b->beginProbe();
        const bool ok = transmit(list, &probe, g.get());
        deferred = b->endProbe() && ok && probe.mPMeasureSize == 0;
    }
    if (runs) *runs = 1;
    if (deferred) {
        // the classical register of each MEASURE node, in program order
        std::vector<int> creg;
        for (QNode *p = list.qList.head->next; p; p = p->next)
            if (p->gateSpecifier == MEASURE_GATE) creg.push_back(static_cast<MeasureNode *>(p)->creg);
        b->beginDeferredMeasure();
        if (!transmit(list, &param, g.get())) return -3;
        if (!b->deferredTerminal() || b->deferredCount() != creg.size()) return -6;
        std::vector<uint64_t> shots;
        if (b->sampleDeferred((size_t)repeat, shots) != qErrorNone) return -6;
        kind = "MEASURE";
        for (uint64_t bits : shots) {
            std::map<size_t, int> regs;                  // as the dispatcher fills mReturnValue
            for (size_t k = 0; k < creg.size(); ++k) regs[(size_t)creg[k]] = (int)((bits >> k) & 1);
            std::stringstream ss;
            for (auto &kv : regs) ss << kv.second;
            std::string bs = ss.str();
            std::reverse(bs.begin(), bs.end());
            res[bs] += 1.0;
        }
        for (auto &kv : res) kv.second /= repeat;
    } else if (!transmit(list, &param, g.get())) {
        return -3;
    } else if (param.mPMeasureSize == 0) {
        if (runs) *runs = repeat;
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

extern "C" int qr_run(const char *path, int backend, int seed, int repeat, char *out, size_t out_len)
{
    return qr_run_ex(path, backend, seed, repeat, 0, out, out_len, nullptr);
}

// The program run once (no shot loop) and the backend's getQState text
// (CPUQuantumGates.cpp:64-82 for the reference CPU backend): backend 0 or
// 1/2 as in qr_run.  Returns the text length, or a negative value.
extern "C" long qr_qstate(const char *path, int backend, int seed, char *out, size_t out_len)
{
    std::string file(path);
    QList list;
    int n = QRunesParser(file, list);
    if (n <= 0 || n > 30) return -1;
    std::unique_ptr<QuantumGates> g;
    if (backend == 0) g.reset(new CPUQuantumGates());
    else if (backend == 1 || backend == 2) g.reset(new B200QuantumGates(backend == 2 ? QS_C64 : QS_C128));
    else return -5;
    QuantumGateParam param;
    param.mQuantumBitNumber = n;
    if (g->initState(&param) != qErrorNone) return -2;
    ref_rng_seed(seed);
    if (!transmit(list, &param, g.get())) return -3;
    std::string s;
    if (!g->getQState(s, &param)) return -3;
    if (s.size() + 1 > out_len) return -(long)(s.size() + 1);
    memcpy(out, s.c_str(), s.size() + 1);
    return (long)s.size();
}
