// rg_server: a serving loop over one pool of arena slots on one GPU (the C ABI rg_server_* in rocketgpu_b200.h).
//
// No counterpart in the reference: the reference steps one BatchSim per call under a process-wide lock
// (src/rocketgpu_cuda.cu:2868-2916). Here many RL clients share one GPU. Each client owns a contiguous range of slots
// in a pool batch (its arenas, created at kickoff like a BatchSim of its own); it submits step requests of 1 to 8
// ticks with the controls of every tick, and polls for the resulting car, ball and env states.
//
// Scheduling. One worker thread owns the pool and its stream. It runs the pool in rounds of one tick: a round steps
// exactly the arenas whose request still has ticks left (the tick kernels skip the others), each reading the
// controls of its own request's current tick (SlotTable in rg_batch.cu). Between rounds the worker
//   * admits queued requests: continuous batching admits every client's next request as soon as its previous one
//     has finished (a request that arrives while others are on the GPU joins at the next round); static batching
//     (the comparison policy) admits a new batch only when the whole previous batch has finished;
//   * starts the result copy of every request whose last tick ran, and completes the requests whose copy is done.
// Arena state stays on the device; only controls go up and results come down. An arena's results depend only on its
// own state and controls: every RNG draw and car id uses the arena's index among its client's arenas and its
// client's kickoff seed, so a client's results are bitwise those of the same arenas stepped alone in a batch.
//
// Admission: the pool's slot count is fixed at open from the HBM budget (budget / device bytes of one slot, capped by
// max_arenas); a client whose arenas do not fit in one free range is refused with RG_BUSY and may retry once others
// close. Nothing on the device waits or spins: each round is an ordinary launch sequence followed by a stream
// synchronisation on the host.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>

namespace {

constexpr int kServerMaxTicks = 8;

__global__ void fill_slots_kernel(int32_t* remaining, int32_t* tick, int32_t* logical, uint64_t* seed, int first,
                                  int n, int32_t value, int set_identity, uint64_t seed_value) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    remaining[first + j] = value;
    tick[first + j] = 0;
    if (set_identity) {
        logical[first + j] = j;
        seed[first + j] = seed_value;
    }
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct ServerRequest {
    int32_t client = -1;
    int32_t ticks = 0;
    int32_t rounds_left = 0;
    enum State { kQueued, kActive, kCopying, kDone } state = kQueued;
    std::vector<rg::CarControls> controls;  // [ticks][arenas * max_cars]
    std::vector<rg_car_state> cars;
    std::vector<rg_ball_state> balls;
    std::vector<rg_env_state> envs;
    cudaEvent_t copied = nullptr;
    double t_submit = 0.0, t_done = 0.0;
};

struct ServerClient {
    int32_t base = 0, n = 0;
    std::deque<int64_t> queue;
    int64_t active = -1;
    rg_car_state* pin_cars = nullptr;  // pinned result staging of the active request
    rg_ball_state* pin_balls = nullptr;
    rg_env_state* pin_envs = nullptr;
    rg::CarControls* pin_controls = nullptr;  // pinned control staging [kServerMaxTicks][n * max_cars]
};

}  // namespace

struct rg_server {
    int device = 0;
    int policy = 0;  // 0 continuous, 1 static
    rg_batch* pool = nullptr;
    cudaStream_t stream = nullptr;
    int32_t capacity = 0;
    int64_t slot_bytes = 0;
    DeviceArray<int32_t> remaining, tick, logical;
    DeviceArray<uint64_t> seed;
    DeviceArray<rg::CarControls> controls;  // [kServerMaxTicks][capacity * max_cars]
    std::vector<int32_t> owner;              // slot -> client id, -1 free
    std::map<int32_t, ServerClient> clients;
    std::map<int64_t, ServerRequest> requests;
    int32_t next_client = 1;
    int64_t next_request = 1;
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stop = false;
    std::string error;
    // statistics
    int64_t rounds = 0, arena_ticks = 0, completed = 0;
    double busy_s = 0.0;
};

namespace {

// Device bytes one arena slot of a pool with `max_cars` car slots takes (the per-arena arrays rg_batch_create
// allocates plus the server's slot tables and control rows).
int64_t server_slot_bytes(int max_cars) {
    const int64_t pairs = static_cast<int64_t>(max_cars) * (max_cars - 1) / 2;
    const int64_t per_arena = sizeof(rg::BallState) + sizeof(rg::EnvState) + sizeof(int32_t) +
                              sizeof(rg::BallWorldScratch) + 34 * sizeof(rg::PadState) + sizeof(rg::Broadphase) +
                              pairs * sizeof(rg::CarCarManifold) + sizeof(rg::ArenaTickSnap) + 2 * sizeof(int32_t) +
                              sizeof(rg::EnvCommand) + sizeof(int64_t) + 3 * sizeof(int32_t) + sizeof(uint64_t);
    const int64_t per_car = sizeof(rg::CarState) + sizeof(rg::WheelRuntime) + sizeof(rg::CarConfig) +
                            (1 + kServerMaxTicks) * sizeof(rg::CarControls) + 1 + sizeof(rg::CarWorldScratch) +
                            sizeof(rg::BallCarScratch) + sizeof(rg::CarTickRecord) + sizeof(rg::CarStage) +
                            sizeof(int32_t) +
                            sizeof(uint64_t);
    return per_arena + static_cast<int64_t>(max_cars) * per_car;
}

void server_launch_round(rg_server* s) {
    rg_batch* b = s->pool;
    CarTickArgs a = car_tick_args(b, s->controls.ptr, b->env_count * b->max_cars);
    a.slots.remaining = s->remaining.ptr;
    a.slots.tick = s->tick.ptr;
    a.slots.logical = s->logical.ptr;
    a.slots.seed = s->seed.ptr;
    const int threads = b->launch_threads;
    const int blocks = (b->env_count + threads - 1) / threads;
    const int ct = b->car_threads;
    const int car_blocks = (b->active_car_count + ct - 1) / ct;
    arena_begin_kernel<<<blocks, threads, 0, s->stream>>>(a, 0);
    if (car_blocks) car_pre_kernel<<<car_blocks, ct, 0, s->stream>>>(a, 0);
    if (car_blocks) car_rays_kernel<<<(4 * b->active_car_count + ct - 1) / ct, ct, 0, s->stream>>>(a, 0);
    if (car_blocks) car_vehicle_kernel<<<car_blocks, ct, 0, s->stream>>>(a, 0);
    arena_finish_kernel<<<blocks, threads, 0, s->stream>>>(a, 0);
    if (car_blocks) car_post_kernel<<<car_blocks, ct, 0, s->stream>>>(a, 0, 0);
    arena_tail_kernel<<<blocks, threads, 0, s->stream>>>(a, 0);
    check(cudaGetLastError(), "serving round launch");
}

// Under s->mu: start the client's next queued request (controls up, its slots armed).
void server_admit(rg_server* s, ServerClient& c) {
    const int64_t id = c.queue.front();
    c.queue.pop_front();
    ServerRequest& r = s->requests.at(id);
    const size_t row = static_cast<size_t>(c.n) * s->pool->max_cars;
    std::memcpy(c.pin_controls, r.controls.data(), r.controls.size() * sizeof(rg::CarControls));
    const size_t stride = static_cast<size_t>(s->capacity) * s->pool->max_cars;
    check(cudaMemcpy2DAsync(s->controls.ptr + static_cast<size_t>(c.base) * s->pool->max_cars,
                            stride * sizeof(rg::CarControls), c.pin_controls, row * sizeof(rg::CarControls),
                            row * sizeof(rg::CarControls), r.ticks, cudaMemcpyHostToDevice, s->stream),
          "request controls");
    fill_slots_kernel<<<(c.n + 127) / 128, 128, 0, s->stream>>>(s->remaining.ptr, s->tick.ptr, s->logical.ptr,
                                                                 s->seed.ptr, c.base, c.n, r.ticks, 0, 0);
    check(cudaGetLastError(), "fill_slots_kernel launch");
    r.state = ServerRequest::kActive;
    r.rounds_left = r.ticks;
    c.active = id;
}

void server_worker(rg_server* s) {
    try {
        check(cudaSetDevice(s->device), "cudaSetDevice");
        std::unique_lock<std::mutex> lk(s->mu);
        while (true) {
            // requests whose results arrived
            for (auto& kv : s->requests) {
                ServerRequest& r = kv.second;
                if (r.state != ServerRequest::kCopying) continue;
                const cudaError_t q = cudaEventQuery(r.copied);
                if (q == cudaErrorNotReady) continue;
                check(q, "result copy");
                ServerClient& c = s->clients.at(r.client);
                std::memcpy(r.cars.data(), c.pin_cars, r.cars.size() * sizeof(rg_car_state));
                std::memcpy(r.balls.data(), c.pin_balls, r.balls.size() * sizeof(rg_ball_state));
                std::memcpy(r.envs.data(), c.pin_envs, r.envs.size() * sizeof(rg_env_state));
                r.state = ServerRequest::kDone;
                r.t_done = now_s();
                c.active = -1;
                ++s->completed;
                s->cv.notify_all();
            }
            // admission
            bool any_busy = false;
            for (auto& kv : s->clients) any_busy = any_busy || kv.second.active >= 0;
            if (s->policy == 0 || !any_busy) {
                for (auto& kv : s->clients) {
                    ServerClient& c = kv.second;
                    if (c.active < 0 && !c.queue.empty()) server_admit(s, c);
                }
            }
            bool any_active = false;
            for (auto& kv : s->clients) {
                if (kv.second.active < 0) continue;
                any_active = any_active || s->requests.at(kv.second.active).state == ServerRequest::kActive;
            }
            if (!any_active) {
                bool copying = false;
                for (auto& kv : s->clients) copying = copying || kv.second.active >= 0;
                if (s->stop && !copying) break;
                if (copying) {
                    lk.unlock();
                    check(cudaStreamSynchronize(s->stream), "serving stream");
                    lk.lock();
                } else {
                    s->cv.wait_for(lk, std::chrono::milliseconds(1));
                }
                continue;
            }
            // one round: every armed arena advances one tick
            const double t0 = now_s();
            server_launch_round(s);
            ++s->rounds;
            for (auto& kv : s->clients) {
                ServerClient& c = kv.second;
                if (c.active < 0) continue;
                ServerRequest& r = s->requests.at(c.active);
                if (r.state != ServerRequest::kActive) continue;
                s->arena_ticks += c.n;
                if (--r.rounds_left > 0) continue;
                const int mc = s->pool->max_cars;
                check(cudaMemcpyAsync(c.pin_cars, s->pool->cars.ptr + static_cast<size_t>(c.base) * mc,
                                      static_cast<size_t>(c.n) * mc * sizeof(rg_car_state), cudaMemcpyDeviceToHost,
                                      s->stream),
                      "result cars");
                check(cudaMemcpyAsync(c.pin_balls, s->pool->balls.ptr + c.base, c.n * sizeof(rg_ball_state),
                                      cudaMemcpyDeviceToHost, s->stream),
                      "result balls");
                check(cudaMemcpyAsync(c.pin_envs, s->pool->envs.ptr + c.base, c.n * sizeof(rg_env_state),
                                      cudaMemcpyDeviceToHost, s->stream),
                      "result envs");
                check(cudaEventRecord(r.copied, s->stream), "result event");
                r.state = ServerRequest::kCopying;
            }
            lk.unlock();
            check(cudaStreamSynchronize(s->stream), "serving round");
            lk.lock();
            s->busy_s += now_s() - t0;
        }
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> g(s->mu);
        s->error = e.what();
        s->cv.notify_all();
    }
}

void server_free_client(rg_server* s, ServerClient& c) {
    if (c.pin_cars) cudaFreeHost(c.pin_cars);
    if (c.pin_balls) cudaFreeHost(c.pin_balls);
    if (c.pin_envs) cudaFreeHost(c.pin_envs);
    if (c.pin_controls) cudaFreeHost(c.pin_controls);
    c.pin_cars = nullptr;
    c.pin_balls = nullptr;
    c.pin_envs = nullptr;
    c.pin_controls = nullptr;
}

// Under s->mu, with the worker idle for this client's slots: the pool's car counts for [base, base + n) and its step
// order.
void server_set_counts(rg_server* s, int base, int n, const int32_t* counts) {
    rg_batch* b = s->pool;
    for (int j = 0; j < n; ++j) {
        b->host_car_count[base + j] = counts ? counts[j] : 0;
        b->pads_live = b->pads_live || (counts && counts[j] > 0);
    }
    rebuild_step_order(b, s->stream);
    check(cudaMemcpyAsync(b->env_car_count.ptr + base, b->host_car_count.data() + base, n * sizeof(int32_t),
                          cudaMemcpyHostToDevice, s->stream),
          "client car counts");
    check(cudaStreamSynchronize(s->stream), "client car counts");
}

}  // namespace

extern "C" {

RG_API int rg_server_open(const rg_server_config* scfg, const rg_sim_config* sim, const rg_arena_layout* layout,
                          int device, rg_server** out) {
    return guard([&] {
        if (!scfg || !sim || !layout || !out) throw std::invalid_argument("null argument");
        if (scfg->policy != 0 && scfg->policy != 1) throw std::invalid_argument("policy must be 0 or 1");
        if (scfg->max_arenas <= 0 && scfg->hbm_budget_bytes <= 0)
            throw std::invalid_argument("give max_arenas or hbm_budget_bytes");
        if (sim->max_cars_per_env <= 0 || sim->max_cars_per_env > 6)
            throw std::invalid_argument("max_cars_per_env must be in [1, 6]");
        // a client's kickoffs run in the pool's slots without the batch's settle entries
        if (sim->kickoff_settled != 0) throw std::invalid_argument("the server takes kickoff_settled = 0");
        std::unique_ptr<rg_server> s(new rg_server);
        s->device = device;
        s->policy = scfg->policy;
        s->slot_bytes = server_slot_bytes(sim->max_cars_per_env);
        int64_t cap = scfg->max_arenas > 0 ? scfg->max_arenas : INT32_MAX;
        if (scfg->hbm_budget_bytes > 0) cap = std::min<int64_t>(cap, scfg->hbm_budget_bytes / s->slot_bytes);
        if (cap <= 0) throw std::invalid_argument("the HBM budget holds no arena slot");
        if (cap > (1 << 24)) throw std::invalid_argument("more than 16M arena slots");
        s->capacity = static_cast<int32_t>(cap);
        rg_sim_config pc = *sim;
        pc.env_count = s->capacity;
        const int rc = rg_batch_create(&pc, layout, device, &s->pool);
        if (rc != 0) throw std::runtime_error(std::string("pool: ") + g_last_error);
        DeviceGuard dg(device);
        check(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        s->remaining.alloc(s->capacity);
        s->tick.alloc(s->capacity);
        s->logical.alloc(s->capacity);
        s->seed.alloc(s->capacity);
        check(cudaMemset(s->remaining.ptr, 0, s->capacity * sizeof(int32_t)), "slot table");
        check(cudaMemset(s->tick.ptr, 0, s->capacity * sizeof(int32_t)), "slot table");
        check(cudaMemset(s->logical.ptr, 0, s->capacity * sizeof(int32_t)), "slot table");
        check(cudaMemset(s->seed.ptr, 0, s->capacity * sizeof(uint64_t)), "slot table");
        s->controls.alloc(static_cast<size_t>(kServerMaxTicks) * s->capacity * sim->max_cars_per_env);
        check(cudaMemset(s->controls.ptr, 0, s->controls.n * sizeof(rg::CarControls)), "slot controls");
        s->owner.assign(s->capacity, -1);
        s->worker = std::thread(server_worker, s.get());
        *out = s.release();
    });
}

RG_API void rg_server_close(rg_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        for (auto& kv : s->clients) kv.second.queue.clear();
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    DeviceGuard dg(s->device);
    for (auto& kv : s->requests)
        if (kv.second.copied) cudaEventDestroy(kv.second.copied);
    for (auto& kv : s->clients) server_free_client(s, kv.second);
    if (s->stream) cudaStreamDestroy(s->stream);
    rg_batch_destroy(s->pool);
    delete s;
}

RG_API int rg_server_client_open(rg_server* s, int32_t arenas, const int32_t* car_counts, const uint8_t* teams,
                                 const rg_car_config* configs, uint64_t kickoff_seed, int32_t* client) {
    return guard([&] {
        if (!s || !car_counts || !client) throw std::invalid_argument("null argument");
        if (arenas <= 0) throw std::invalid_argument("arenas must be positive");
        const int mc = s->pool->max_cars;
        for (int j = 0; j < arenas; ++j)
            if (car_counts[j] < 0 || car_counts[j] > mc)
                throw std::out_of_range("car count out of range [0, max_cars_per_env]");
        for (int j = 0; teams && j < arenas * mc; ++j)
            if (teams[j] > 1) throw std::invalid_argument("team must be 0 (blue) or 1 (orange)");
        for (int j = 0; configs && j < arenas * mc; ++j)
            if (configs[j].three_wheels) throw std::invalid_argument("three-wheel car configs are not supported");
        std::unique_lock<std::mutex> lk(s->mu);
        if (!s->error.empty()) throw std::runtime_error("server failed: " + s->error);
        DeviceGuard dg(s->device);
        // the worker launches rounds only under the lock; wait for the one in flight before touching the pool
        check(cudaStreamSynchronize(s->stream), "serving stream");
        int base = -1;
        for (int i = 0, run = 0; i < s->capacity; ++i) {
            run = s->owner[i] < 0 ? run + 1 : 0;
            if (run == arenas) {
                base = i - arenas + 1;
                break;
            }
        }
        if (base < 0) throw ServerBusy("no free range of " + std::to_string(arenas) + " arena slots (capacity " +
                                       std::to_string(s->capacity) + ")");
        const int32_t id = s->next_client++;
        ServerClient c;
        c.base = base;
        c.n = arenas;
        const size_t cars = static_cast<size_t>(arenas) * mc;
        check(cudaMallocHost(&c.pin_cars, cars * sizeof(rg_car_state)), "pinned results");
        check(cudaMallocHost(&c.pin_balls, arenas * sizeof(rg_ball_state)), "pinned results");
        check(cudaMallocHost(&c.pin_envs, arenas * sizeof(rg_env_state)), "pinned results");
        check(cudaMallocHost(&c.pin_controls, kServerMaxTicks * cars * sizeof(rg::CarControls)), "pinned controls");
        rg_batch* b = s->pool;
        // the client's arenas as a fresh batch of its own: default cars, its teams and bodies, then its kickoff
        {
            rg_car_state c0;
            rg_default_car_state(&c0);
            rg_car_config k0;
            rg_default_car_config(&k0);
            std::vector<rg_car_state> cs(cars, c0);
            std::vector<rg_car_config> ks(cars, k0);
            if (configs) std::memcpy(ks.data(), configs, cars * sizeof(rg_car_config));
            std::vector<uint8_t> ts(cars, 0);
            if (teams) std::memcpy(ts.data(), teams, cars);
            std::vector<rg::WheelRuntime> ws(cars, rg::wheel_runtime_default());
            std::vector<rg_ball_state> bs(arenas);
            std::vector<rg_env_state> es(arenas);
            for (auto& x : bs) rg_default_ball_state(&x);
            for (auto& x : es) rg_default_env_state(&x);
            const size_t off = static_cast<size_t>(base) * mc;
            cudaStream_t st = s->stream;
            check(cudaMemcpyAsync(b->cars.ptr + off, cs.data(), cars * sizeof(rg_car_state), cudaMemcpyHostToDevice,
                                  st),
                  "client cars");
            check(cudaMemcpyAsync(b->car_cfgs.ptr + off, ks.data(), cars * sizeof(rg_car_config),
                                  cudaMemcpyHostToDevice, st),
                  "client configs");
            check(cudaMemcpyAsync(b->teams.ptr + off, ts.data(), cars, cudaMemcpyHostToDevice, st), "client teams");
            check(cudaMemcpyAsync(b->wheels.ptr + off, ws.data(), cars * sizeof(rg::WheelRuntime),
                                  cudaMemcpyHostToDevice, st),
                  "client wheels");
            check(cudaMemcpyAsync(b->balls.ptr + base, bs.data(), arenas * sizeof(rg_ball_state),
                                  cudaMemcpyHostToDevice, st),
                  "client balls");
            check(cudaMemcpyAsync(b->envs.ptr + base, es.data(), arenas * sizeof(rg_env_state), cudaMemcpyHostToDevice,
                                  st),
                  "client envs");
            check(cudaMemsetAsync(b->ball_world.ptr + base, 0, arenas * sizeof(rg::BallWorldScratch), st),
                  "client contacts");
            check(cudaStreamSynchronize(st), "client state");
        }
        server_set_counts(s, base, arenas, car_counts);
        fill_slots_kernel<<<(arenas + 127) / 128, 128, 0, s->stream>>>(s->remaining.ptr, s->tick.ptr, s->logical.ptr,
                                                                        s->seed.ptr, base, arenas, 0, 1,
                                                                        kickoff_seed);
        check(cudaGetLastError(), "fill_slots_kernel launch");
        // BatchSim's constructor resets to kickoff with seed 0; the client's own reset follows (reference
        // src/rocketgpu.cpp:1281, 2085-2132)
        CarTickArgs a = car_tick_args(b, nullptr, 0);
        a.pads = b->pads.ptr;
        for (uint64_t seed : {static_cast<uint64_t>(0), kickoff_seed}) {
            reset_kickoff_kernel<<<(arenas + 63) / 64, 64, 0, s->stream>>>(a, b->teams.ptr, b->controls.ptr, seed, base,
                                                                            arenas);
            check(cudaGetLastError(), "client kickoff");
        }
        check(cudaStreamSynchronize(s->stream), "client open");
        for (int j = 0; j < arenas; ++j) s->owner[base + j] = id;
        s->clients.emplace(id, std::move(c));
        *client = id;
    });
}

RG_API int rg_server_client_close(rg_server* s, int32_t client) {
    return guard([&] {
        if (!s) throw std::invalid_argument("null argument");
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->clients.find(client);
        if (it == s->clients.end()) throw std::out_of_range("unknown client");
        ServerClient& c = it->second;
        c.queue.clear();
        // an admitted request finishes its ticks (its arenas are on the GPU); then the slots are free
        s->cv.wait(lk, [&] { return c.active < 0 || !s->error.empty(); });
        for (auto r = s->requests.begin(); r != s->requests.end();) {
            if (r->second.client == client) {
                if (r->second.copied) cudaEventDestroy(r->second.copied);
                r = s->requests.erase(r);
            } else {
                ++r;
            }
        }
        DeviceGuard dg(s->device);
        check(cudaStreamSynchronize(s->stream), "serving stream");
        server_set_counts(s, c.base, c.n, nullptr);
        for (int j = 0; j < c.n; ++j) s->owner[c.base + j] = -1;
        server_free_client(s, c);
        s->clients.erase(it);
    });
}

RG_API int rg_server_submit(rg_server* s, int32_t client, int32_t ticks, const rg_car_controls* host_controls,
                            int64_t* request) {
    return guard([&] {
        if (!s || !host_controls || !request) throw std::invalid_argument("null argument");
        if (ticks < 1 || ticks > kServerMaxTicks) throw std::invalid_argument("ticks must be in [1, 8]");
        std::lock_guard<std::mutex> g(s->mu);
        if (!s->error.empty()) throw std::runtime_error("server failed: " + s->error);
        if (s->stop) throw std::runtime_error("server is closing");
        auto it = s->clients.find(client);
        if (it == s->clients.end()) throw std::out_of_range("unknown client");
        const ServerClient& c = it->second;
        const size_t cars = static_cast<size_t>(c.n) * s->pool->max_cars;
        ServerRequest r;
        r.client = client;
        r.ticks = ticks;
        r.controls.resize(cars * ticks);
        std::memcpy(r.controls.data(), host_controls, r.controls.size() * sizeof(rg::CarControls));
        r.cars.resize(cars);
        r.balls.resize(c.n);
        r.envs.resize(c.n);
        DeviceGuard dg(s->device);
        check(cudaEventCreateWithFlags(&r.copied, cudaEventDisableTiming), "cudaEventCreate");
        r.t_submit = now_s();
        const int64_t id = s->next_request++;
        s->requests.emplace(id, std::move(r));
        it->second.queue.push_back(id);
        *request = id;
        s->cv.notify_all();
    });
}

RG_API int rg_server_poll(rg_server* s, int64_t request, int32_t wait_ms, rg_car_state* cars_out,
                          rg_ball_state* balls_out, rg_env_state* envs_out, int32_t* done, double* latency_s) {
    return guard([&] {
        if (!s || !done) throw std::invalid_argument("null argument");
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->requests.find(request);
        if (it == s->requests.end()) throw std::out_of_range("unknown request");
        auto finished = [&] { return it->second.state == ServerRequest::kDone || !s->error.empty(); };
        if (!finished() && wait_ms > 0) s->cv.wait_for(lk, std::chrono::milliseconds(wait_ms), finished);
        if (!s->error.empty()) throw std::runtime_error("server failed: " + s->error);
        ServerRequest& r = it->second;
        *done = r.state == ServerRequest::kDone ? 1 : 0;
        if (!*done) return;
        if (cars_out) std::memcpy(cars_out, r.cars.data(), r.cars.size() * sizeof(rg_car_state));
        if (balls_out) std::memcpy(balls_out, r.balls.data(), r.balls.size() * sizeof(rg_ball_state));
        if (envs_out) std::memcpy(envs_out, r.envs.data(), r.envs.size() * sizeof(rg_env_state));
        if (latency_s) *latency_s = r.t_done - r.t_submit;
        DeviceGuard dg(s->device);
        cudaEventDestroy(r.copied);
        s->requests.erase(it);
    });
}

RG_API int rg_server_get_stats(rg_server* s, rg_server_stats* out) {
    return guard([&] {
        if (!s || !out) throw std::invalid_argument("null argument");
        std::lock_guard<std::mutex> g(s->mu);
        out->capacity = s->capacity;
        int64_t used = 0;
        for (int32_t o : s->owner) used += o >= 0;
        out->used = used;
        out->slot_bytes = s->slot_bytes;
        out->clients = static_cast<int64_t>(s->clients.size());
        out->rounds = s->rounds;
        out->arena_ticks = s->arena_ticks;
        out->completed = s->completed;
        out->busy_s = s->busy_s;
    });
}

}  // extern "C"
