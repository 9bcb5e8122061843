// A serving loop over the batched scorer: requests (each a batch of pairs under a Scoring) arrive at any
// time, wait in a queue, and are admitted first in first out as a worker slot and device memory free up;
// a slot that frees up takes the head of the queue with every request queued behind it that shares its
// Scoring and mode, as one device call (continuous batching).
// Each slot is a context of its own on the device (its stream and the device buffers it keeps between
// requests), so admitted requests run at once and their kernels overlap on the GPU; a request's result
// is the same whether it runs alone or beside others, as no slot shares a buffer with another.
//
// Device memory is budgeted: a request is admitted only when every slot's resident buffers, with the
// admitting slot grown to the request's estimate, fit the budget; idle slots give their buffers back when
// a request would not otherwise fit, and a request that cannot fit an empty device is refused.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point origin) {
    return std::chrono::duration<double>(Clock::now() - origin).count();
}

struct Request {
    int64_t ticket = 0;
    int64_t pairs = 0;
    std::vector<char> letters;
    std::vector<int64_t> offsets;
    std::string alphabet;
    std::vector<int8_t> table;
    int64_t opening = 0, extension = 0;
    dinara_mode mode{};
    std::vector<int32_t> scores;
    std::vector<int64_t> statuses;
    int64_t code = 0;
    int64_t estimate = 0;  // device bytes the request's run may hold
    double submitted = 0, admitted = 0, finished = 0;
    bool done = false;
};

// Device bytes a context holds in its buffers and its partner's (the second stream a large batch's units
// alternate onto).
int64_t resident_bytes(dinara_gpu *g) {
    int64_t total = 0;
    g->for_each_buffer([&](const dinara::DeviceBuffer &b) { total += int64_t(b.bytes); });
    if (g->partner) total += resident_bytes(g->partner);
    return total;
}

// Gives a context's device buffers (and its partner's) back to the device's pool, each ordered after its
// own stream's work.
void release_buffers(dinara_gpu *g) {
    cudaSetDevice(g->device);
    {
        dinara::AllocationScope scope(g->stream);
        g->for_each_buffer([](dinara::DeviceBuffer &b) { b.release(); });
    }
    if (g->partner) release_buffers(g->partner);
}

// What a request's scores may hold on the device: its letters and their packed copy, per-pair shapes,
// keys, orders and results, and the carried columns of pairs wider than one strip (a group's slot as long
// as the tallest pair, for every group the widest launch runs).
int64_t estimate_bytes(const Request &r, int multiprocessors) {
    int64_t letters = r.offsets.empty() ? 0 : r.offsets.back() - r.offsets.front();
    int64_t max_rows = 0, max_columns = 0;
    for (int64_t p = 0; p < r.pairs; ++p) {
        max_rows = std::max(max_rows, r.offsets[size_t(2 * p + 1)] - r.offsets[size_t(2 * p)]);
        max_columns = std::max(max_columns, r.offsets[size_t(2 * p + 2)] - r.offsets[size_t(2 * p + 1)]);
    }
    int64_t bytes = 2 * letters + 160 * r.pairs + (int64_t(64) << 20);
    if (max_columns > 256) bytes += int64_t(multiprocessors) * 2 * 8 * (max_rows + 1) * 8;
    return bytes;
}

// Whether two requests can share one device call: the same Scoring and the same mode.
bool compatible(const Request &a, const Request &b) {
    return a.alphabet == b.alphabet && a.table == b.table && a.opening == b.opening && a.extension == b.extension &&
           std::memcmp(&a.mode, &b.mode, sizeof a.mode) == 0;
}

// Pairs one merged device call may hold.
constexpr int64_t kMergePairs = int64_t(1) << 20;

}  // namespace

struct dinara_server {
    dinara_gpu *owner = nullptr;
    std::vector<dinara_gpu *> slots;
    std::vector<bool> busy;
    // Bytes each slot holds as last seen while it was idle, or its running request's estimate if larger;
    // read only under the lock, so no slot's buffers are read while its worker grows them.
    std::vector<int64_t> held;
    std::vector<std::thread> workers;
    std::mutex lock;
    std::condition_variable work, finished;
    std::deque<Request *> queue;
    std::map<int64_t, Request *> requests;
    int64_t budget = 0;
    int64_t next_ticket = 1;
    bool stopping = false;
    Clock::time_point origin = Clock::now();
    int64_t admitted = 0, completed = 0, refused = 0, pairs_done = 0, calls = 0;

    // Bytes every slot holds, the slot `k` counted at least `grown` (its request's estimate).
    int64_t projected(size_t k, int64_t grown) {
        int64_t total = 0;
        for (size_t j = 0; j < slots.size(); ++j) total += j == k ? std::max(held[j], grown) : held[j];
        return total;
    }

    void release(size_t j) {
        release_buffers(slots[j]);
        held[j] = 0;
    }

    // Scores a batch of compatible requests in one device call on a slot, each request's results into it.
    static int64_t run_batch(dinara_gpu *slot, const std::vector<Request *> &batch, int64_t pairs) {
        Request &first = *batch.front();
        dinara_scoring scoring{first.alphabet.data(), int64_t(first.alphabet.size()), first.table.data(),
                               first.opening, first.extension};
        for (Request *q : batch) {
            q->scores.assign(size_t(std::max<int64_t>(q->pairs, 1)), 0);
            q->statuses.assign(size_t(std::max<int64_t>(q->pairs, 1)), 0);
        }
        if (batch.size() == 1)
            return dinara_gpu_scores_tape(slot, first.pairs, first.letters.data(), first.offsets.data(), &scoring,
                                          &first.mode, first.scores.data(), first.statuses.data());
        std::vector<char> letters;
        std::vector<int64_t> offsets{0};
        offsets.reserve(size_t(2 * pairs + 1));
        for (const Request *q : batch) {
            const int64_t base = offsets.back();
            const int64_t length = q->offsets.empty() ? 0 : q->offsets.back();
            letters.insert(letters.end(), q->letters.begin(), q->letters.begin() + length);
            for (int64_t j = 1; j <= 2 * q->pairs; ++j) offsets.push_back(base + q->offsets[size_t(j)]);
        }
        letters.push_back(0);
        std::vector<int32_t> scores(size_t(std::max<int64_t>(pairs, 1)));
        std::vector<int64_t> statuses(size_t(std::max<int64_t>(pairs, 1)));
        const int64_t code = dinara_gpu_scores_tape(slot, pairs, letters.data(), offsets.data(), &scoring, &first.mode,
                                                    scores.data(), statuses.data());
        int64_t at = 0;
        for (Request *q : batch) {
            std::copy(scores.begin() + at, scores.begin() + at + q->pairs, q->scores.begin());
            std::copy(statuses.begin() + at, statuses.begin() + at + q->pairs, q->statuses.begin());
            at += q->pairs;
        }
        return code;
    }

    void worker(size_t k) {
        std::unique_lock<std::mutex> hold(lock);
        for (;;) {
            work.wait(hold, [&] { return stopping || !queue.empty(); });
            if (stopping && queue.empty()) return;
            Request *r = queue.front();
            if (projected(k, r->estimate) > budget) {
                // Idle slots give their buffers back before the request is held back.
                for (size_t j = 0; j < slots.size(); ++j)
                    if (!busy[j] && j != k && held[j] > 0) release(j);
                if (projected(k, r->estimate) > budget) {
                    bool anyone_busy = false;
                    for (size_t j = 0; j < slots.size(); ++j) anyone_busy = anyone_busy || busy[j];
                    if (!anyone_busy) {
                        release(k);
                        if (r->estimate > budget) {
                            // Past the whole budget: refused, as the reference refuses what its device
                            // cannot hold (common.mojo:211-218).
                            queue.pop_front();
                            r->code = DINARA_OUT_OF_MEMORY;
                            r->done = true;
                            r->finished = seconds_since(origin);
                            ++refused;
                            finished.notify_all();
                            continue;
                        }
                    } else {
                        // Wait for a running request to finish and free its memory.
                        finished.wait_for(hold, std::chrono::milliseconds(50));
                        continue;
                    }
                }
            }
            queue.pop_front();
            // Continuous batching: the requests queued behind this one that share its Scoring and mode
            // join it in one device call, as far as the pair cap and the memory budget allow.
            std::vector<Request *> batch{r};
            int64_t batch_pairs = r->pairs, batch_estimate = r->estimate;
            while (!queue.empty() && compatible(*queue.front(), *r) &&
                   batch_pairs + queue.front()->pairs <= kMergePairs &&
                   projected(k, batch_estimate + queue.front()->estimate) <= budget) {
                batch.push_back(queue.front());
                batch_pairs += queue.front()->pairs;
                batch_estimate += queue.front()->estimate;
                queue.pop_front();
            }
            busy[k] = true;
            held[k] = std::max(held[k], batch_estimate);
            const double now = seconds_since(origin);
            for (Request *q : batch) q->admitted = now;
            admitted += int64_t(batch.size());
            ++calls;
            hold.unlock();
            const int64_t code = run_batch(slots[k], batch, batch_pairs);
            const int64_t now_held = resident_bytes(slots[k]);
            hold.lock();
            held[k] = now_held;
            const double end = seconds_since(origin);
            for (Request *q : batch) {
                q->code = code;
                q->done = true;
                q->finished = end;
                pairs_done += q->pairs;
            }
            busy[k] = false;
            completed += int64_t(batch.size());
            finished.notify_all();
            work.notify_all();
        }
    }
};

extern "C" {

dinara_server *dinara_server_new(dinara_gpu *gpu, const dinara_server_options *options) {
    if (!gpu) return nullptr;
    dinara_server *server = new dinara_server();
    server->owner = gpu;
    const int64_t slots = options && options->slots > 0 ? std::min<int64_t>(options->slots, 32) : 4;
    server->budget = options && options->device_bytes > 0 ? options->device_bytes : (int64_t(40) << 30);
    for (int64_t k = 0; k < slots; ++k) {
        dinara_gpu *slot = dinara_gpu_new(gpu->device);
        if (!slot) {
            for (auto *s : server->slots) dinara_gpu_free(s);
            gpu->error = "a serving slot's context could not be opened";
            delete server;
            return nullptr;
        }
        server->slots.push_back(slot);
        server->busy.push_back(false);
        server->held.push_back(0);
    }
    for (size_t k = 0; k < server->slots.size(); ++k) server->workers.emplace_back([server, k] { server->worker(k); });
    return server;
}

void dinara_server_free(dinara_server *server) {
    if (!server) return;
    {
        std::lock_guard<std::mutex> hold(server->lock);
        server->stopping = true;
    }
    server->work.notify_all();
    for (auto &t : server->workers) t.join();
    for (auto *s : server->slots) dinara_gpu_free(s);
    for (auto &entry : server->requests) delete entry.second;
    delete server;
}

int64_t dinara_server_submit(dinara_server *server, int64_t pairs, const char *letters, const int64_t *offsets,
                             const dinara_scoring *scoring, const dinara_mode *mode, int64_t *ticket) {
    if (!server || !ticket || !scoring || !scoring->alphabet || !scoring->table) return DINARA_INVALID_MODE;
    if (pairs < 0 || (pairs > 0 && !offsets)) return DINARA_INVALID_LENGTH;
    for (int64_t k = 0; k < 2 * pairs; ++k)
        if (offsets[k + 1] < offsets[k]) return DINARA_INVALID_LENGTH;
    Request *r = new Request();
    r->pairs = pairs;
    if (pairs > 0) {
        r->letters.assign(letters + offsets[0], letters + offsets[2 * pairs]);
        r->offsets.resize(size_t(2 * pairs + 1));
        for (int64_t k = 0; k <= 2 * pairs; ++k) r->offsets[size_t(k)] = offsets[k] - offsets[0];
    }
    r->letters.push_back(0);
    r->alphabet.assign(scoring->alphabet, size_t(std::max<int64_t>(scoring->alphabet_size, 0)));
    r->table.assign(scoring->table, scoring->table + std::max<int64_t>(scoring->alphabet_size, 0) *
                                                          std::max<int64_t>(scoring->alphabet_size, 0));
    r->opening = scoring->opening;
    r->extension = scoring->extension;
    if (mode) r->mode = *mode;
    r->estimate = estimate_bytes(*r, server->owner->multiprocessors);
    std::lock_guard<std::mutex> hold(server->lock);
    r->ticket = server->next_ticket++;
    r->submitted = seconds_since(server->origin);
    server->requests[r->ticket] = r;
    server->queue.push_back(r);
    *ticket = r->ticket;
    server->work.notify_one();
    return 0;
}

int64_t dinara_server_wait(dinara_server *server, int64_t ticket, int64_t timeout_ms, int32_t *scores,
                           int64_t *statuses, dinara_request_timing *timing) {
    if (!server) return DINARA_INVALID_MODE;
    std::unique_lock<std::mutex> hold(server->lock);
    auto found = server->requests.find(ticket);
    if (found == server->requests.end()) return DINARA_INVALID_MODE;
    Request *r = found->second;
    // A bounded wait: the caller learns of a stalled request instead of waiting for good.
    const bool ready = server->finished.wait_for(hold, std::chrono::milliseconds(std::max<int64_t>(timeout_ms, 0)),
                                                 [&] { return r->done; });
    if (!ready) return DINARA_DEVICE_TIMEOUT;
    // A refused request never ran and holds no results: nothing is written for it.
    const bool ran = r->scores.size() >= size_t(r->pairs) && r->statuses.size() >= size_t(r->pairs);
    if (ran && scores && r->pairs > 0) std::memcpy(scores, r->scores.data(), size_t(r->pairs) * sizeof(int32_t));
    if (ran && statuses && r->pairs > 0)
        std::memcpy(statuses, r->statuses.data(), size_t(r->pairs) * sizeof(int64_t));
    if (timing) {
        timing->submitted = r->submitted;
        timing->admitted = r->admitted;
        timing->finished = r->finished;
        timing->pairs = r->pairs;
        timing->device_bytes = r->estimate;
    }
    const int64_t code = r->code;
    server->requests.erase(found);
    delete r;
    return code;
}

int64_t dinara_server_stats(dinara_server *server, dinara_server_stats_t *stats) {
    if (!server || !stats) return DINARA_INVALID_MODE;
    std::lock_guard<std::mutex> hold(server->lock);
    stats->queued = int64_t(server->queue.size());
    stats->admitted = server->admitted;
    stats->completed = server->completed;
    stats->refused = server->refused;
    stats->pairs_done = server->pairs_done;
    int64_t resident = 0, running = 0;
    for (size_t k = 0; k < server->slots.size(); ++k) {
        resident += server->held[k];
        running += server->busy[k] ? 1 : 0;
    }
    stats->resident_bytes = resident;
    stats->running = running;
    stats->budget_bytes = server->budget;
    stats->clock = seconds_since(server->origin);
    stats->calls = server->calls;
    return 0;
}

}  // extern "C"
