// mailbox.cpp - TEST HARNESS for the sharded driver's paths to a partner
// shard held by another qs_sharded (another process in a multi-GPU job), on
// one GPU: one host thread per shard, each with its own qs_sharded holding
// that one shard, and either
//   * mailbox_run: an exchange function that meets the partner's thread at a
//     host mailbox and copies the partner's packed half into this shard's
//     receive buffer, or
//   * peer_run: every other shard registered as a peer (qs_sharded_set_peer,
//     its device address standing in for a peer GPU's or an IPC-mapped
//     buffer) and a pairwise host barrier; each side's swap kernel trades its
//     half of the rows in place.
// Only host threads wait (on a mutex and condition variable); no kernel waits
// on another: the two sides' swap kernels touch disjoint element pairs.
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "qpanda_b200.h"

namespace {

struct Slot {
    const void *send = nullptr;
    size_t bytes = 0;
    long long round = 0;          // exchanges posted by this shard
    long long taken = 0;          // exchanges of this shard its partner has copied
};

struct Mailbox {
    std::mutex mu;
    std::condition_variable cv;
    std::vector<Slot> slot;
};

int exchange(void *ctx, int shard, int partner, const void *send, void *recv, size_t bytes, void *)
{
    Mailbox &M = *static_cast<Mailbox *>(ctx);
    std::unique_lock<std::mutex> lk(M.mu);
    Slot &me = M.slot[shard], &pa = M.slot[partner];
    me.send = send;
    me.bytes = bytes;
    const long long round = ++me.round;
    M.cv.notify_all();
    if (!M.cv.wait_for(lk, std::chrono::seconds(60), [&] { return pa.round >= round; })) return 1;
    if (pa.bytes != bytes) return 2;
    const void *src = pa.send;
    lk.unlock();
    const cudaError_t e = cudaMemcpy(recv, src, bytes, cudaMemcpyDeviceToDevice);
    lk.lock();
    ++pa.taken;                   // the partner may reuse its send buffer
    M.cv.notify_all();
    if (!M.cv.wait_for(lk, std::chrono::seconds(60), [&] { return me.taken >= round; })) return 3;
    return e == cudaSuccess ? 0 : 4;
}

}  // namespace

// Run `gates` on an n-qubit state over 2^g shards, one thread and one
// qs_sharded per shard.  out: 2^g x 2^(n-g) amplitudes of dtype (host),
// shard by shard; pos: n entries.  Returns 0 or the first failing status.
extern "C" int mailbox_run(int n, int g, int dtype, const qs_gate *gates, size_t count, void *out, int *pos,
                           size_t *swaps)
{
    const int shards = 1 << g;
    Mailbox M;
    M.slot.resize(shards);
    std::vector<int> rc(shards, 0);
    const size_t shard_bytes = ((size_t)1 << (n - g)) * (dtype == QS_C64 ? 8 : 16);
    std::vector<std::thread> th;
    for (int r = 0; r < shards; ++r)
        th.emplace_back([&, r] {
            cudaSetDevice(0);
            qs_sharded *S = nullptr;
            int e = qs_sharded_create(n, g, dtype, &r, 1, exchange, &M, &S);
            if (!e) e = qs_sharded_apply(S, gates, count);
            qs_state *s = nullptr;
            if (!e) e = qs_sharded_shard(S, r, &s);
            if (!e) e = qs_get_state(s, static_cast<char *>(out) + r * shard_bytes, dtype);
            if (!e && r == 0) e = qs_sharded_positions(S, pos);
            if (!e && r == 0) e = qs_sharded_info(S, swaps, nullptr);
            qs_sharded_destroy(S);
            rc[r] = e;
        });
    for (auto &t : th) t.join();
    for (int r = 0; r < shards; ++r)
        if (rc[r]) return rc[r];
    return 0;
}

namespace {

struct Rendezvous {
    std::mutex mu;
    std::condition_variable cv;
    std::vector<std::vector<long long>> calls;    // calls[a][b]: barrier calls of shard a with partner b
    int ready = 0;
    std::vector<void *> amp;                      // each shard's device address
};

int barrier(void *ctx, int shard, int partner)
{
    Rendezvous &R = *static_cast<Rendezvous *>(ctx);
    std::unique_lock<std::mutex> lk(R.mu);
    const long long k = ++R.calls[shard][partner];
    R.cv.notify_all();
    return R.cv.wait_for(lk, std::chrono::seconds(60), [&] { return R.calls[partner][shard] >= k; }) ? 0 : 1;
}

}  // namespace

// As mailbox_run, with every swap between two threads' shards done by peer
// swaps (qs_sharded_set_peer) instead of an exchange function.
extern "C" int peer_run(int n, int g, int dtype, const qs_gate *gates, size_t count, void *out, int *pos,
                        size_t *swaps, size_t *bytes)
{
    const int shards = 1 << g;
    Rendezvous R;
    R.calls.assign(shards, std::vector<long long>(shards, 0));
    R.amp.assign(shards, nullptr);
    std::vector<int> rc(shards, 0);
    const size_t shard_bytes = ((size_t)1 << (n - g)) * (dtype == QS_C64 ? 8 : 16);
    std::vector<std::thread> th;
    for (int r = 0; r < shards; ++r)
        th.emplace_back([&, r] {
            cudaSetDevice(0);
            qs_sharded *S = nullptr;
            qs_state *s = nullptr;
            void *mine = nullptr;
            int e = qs_sharded_create(n, g, dtype, &r, 1, nullptr, nullptr, &S);
            if (!e) e = qs_sharded_shard(S, r, &s);
            if (!e) e = qs_device_ptr(s, &mine);
            {
                std::unique_lock<std::mutex> lk(R.mu);
                R.amp[r] = mine;
                ++R.ready;
                R.cv.notify_all();
                if (!R.cv.wait_for(lk, std::chrono::seconds(60), [&] { return R.ready == shards; }) && !e) e = 5;
            }
            for (int p = 0; p < shards && !e; ++p)
                if (p != r) e = R.amp[p] ? qs_sharded_set_peer(S, p, R.amp[p], barrier, &R) : 6;
            if (!e) e = qs_sharded_apply(S, gates, count);
            if (!e) e = qs_get_state(s, static_cast<char *>(out) + r * shard_bytes, dtype);
            if (!e && r == 0) e = qs_sharded_positions(S, pos);
            if (!e && r == 0) e = qs_sharded_info(S, swaps, bytes);
            qs_sharded_destroy(S);
            rc[r] = e;
        });
    for (auto &t : th) t.join();
    for (int r = 0; r < shards; ++r)
        if (rc[r]) return rc[r];
    return 0;
}
