// The serving loop in C++ (fx_server_*): requests that arrive over time, solved on one device with
// continuous batching, latency measured by the host's steady clock from arrival to the result.
//
// A request is prepared by its caller (the mesh compiled, the resident state made) and added with
// its arrival time: a static solve K x = b on a resident fx_force (which several requests may
// share), or a quasi-static J2 load path on a compiled mesh (triangular load cycles, Newton per step).
// fx_server_run serves them:
//   - a request becomes visible at its arrival (real time) or at once;
//   - static solves are admitted, in arrival order, into the batched engine (fx_engine_*) while
//     the footprint of the admitted requests (their meshes' device bytes) fits the budget and the
//     engine has a slot and a range of chunks; the engine advances every admitted solve in ticks of 8
//     inner iterations (one batched launch per operator apply for all of them; each solve in its own
//     phase), so requests that arrive while others run join at the next tick;
//   - J2 load paths run in cohorts on up to max_lanes lanes: while a lane is free, the waiting
//     requests with the head's load path (in arrival order, up to max_cohort, while the footprint
//     fits) become one batched Newton (fx_nbatch_*: one combined mesh, per-instance Newton and CG on
//     the device) on it. A lane is a host thread with its own stream that steps its cohort through
//     the load path, so the cohorts' launches and host waits overlap the engine's ticks (run by the
//     loop's own thread) on the device. A running cohort takes no new members (its combined mesh is
//     fixed), so J2 requests that arrive while it runs start the next cohort on another lane;
//   - finished requests are retired and their results kept.
// Each request's arithmetic is that of the request alone, so its result is bit for bit the same
// alone and in any mix: a static solve as the engine's (the FX_SOLVER_IR solve of its mesh), a J2
// path as fx_nbatch_step's (the single-mesh Newton path, tests/test_gpu_nbatch.py).
// No counterpart in the reference, which runs one analysis per process.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

#include "force.hpp"
#include "host.hpp"

namespace fx {
namespace {

template <class F>
int guard(F&& f) {
  try {
    f();
    return FX_OK;
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_error(e.what());
    return FX_E_INVALID;
  }
}

// fext = f * factor (one rounding, as a tensor product by a float)
__global__ void k_scaled(const double* __restrict__ f, double factor, double* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = f[i] * factor;
}
// hist[j] = u[idx[j]]
__global__ void k_pick(const double* __restrict__ u, const int64_t* __restrict__ idx, int n, double* __restrict__ hist) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) hist[j] = u[idx[j]];
}

// With no engine slot in use, the loop polls its lanes and the arrivals at this interval (seconds).
constexpr double kPoll = 2e-4;

void ck(int rc, const char* what) {
  if (rc != FX_OK) throw Error(rc, std::string(what) + ": " + fx_last_error());
}

// Load factors of `cycles` triangular cycles 0 -> 1 -> -1 -> 0, `spc` steps each (step k at
// t = k / spc, phase t mod 1).
std::vector<double> cyclic_factors(int cycles, int spc) {
  std::vector<double> f;
  for (int k = 1; k <= cycles * spc; ++k) {
    const double t = static_cast<double>(k) / static_cast<double>(spc);
    const double ph = std::fmod(t, 1.0);
    f.push_back(ph <= 0.25 ? 4 * ph : ph <= 0.75 ? 2 - 4 * ph : 4 * ph - 4);
  }
  return f;
}

struct Request {
  int64_t id = 0;
  int kind = 0;  // 0 static solve, 1 J2 load path
  double arrival = 0.0;
  // static
  fx_force* f = nullptr;
  std::vector<double> b;
  // J2
  fx_mesh mesh{};
  std::vector<double> unit;  // the load at factor 1 (host, num_equations)
  int64_t monitor = 0;
  int cycles = 1, spc = 8;
  double tol = 1e-6, cg_rtol = 1e-12;
  int max_newton = 25, cg_max_it = 20000;
  // results
  int64_t n = 0;
  int64_t footprint = 0;
  double admitted = -1.0, done = -1.0;
  std::vector<double> x;
  fx_solve_result res{};
  std::vector<double> hist;     // J2: the monitored displacement after each step
  std::vector<int32_t> newton;  // J2: Newton solves per step
};

// Device bytes of one J2 instance in a cohort: element maps and slots (8 nodes, 24 equations, 24
// slot values, the parameter), the material state of 8 points (two 13-value states and an 8-value
// tangent), and about 20 vectors of its equations.
int64_t j2_footprint(const fx_mesh& m) {
  const int64_t per_element = 4 * (8 + 24 + 1) + 8 * 24 + 8 * 8 * (2 * 13 + 8);
  return static_cast<int64_t>(m.padded) * per_element + 8 * 20 * static_cast<int64_t>(m.num_equations);
}

struct Cohort {
  fx_nbatch* nb = nullptr;
  cudaStream_t st = nullptr;
  std::vector<size_t> members;
  std::vector<double> factors;
  std::vector<int64_t> offsets, neq;
  int k = 0;
  DeviceArray<double> F, fext, u, hist;
  DeviceArray<int64_t> idx;
  std::vector<char> conv;
  std::vector<std::vector<int32_t>> newton;
  int64_t footprint = 0;
  // the batched Newton, its stream and device vectors (the lane's thread frees them when the path ends)
  void release() {
    if (nb) fx_nbatch_destroy(nb);
    nb = nullptr;
    F.release();
    fext.release();
    u.release();
    hist.release();
    idx.release();
    if (st) cudaStreamDestroy(st);
    st = nullptr;
  }
  ~Cohort() { release(); }
};

// A lane: the thread that steps one cohort through its load path. state 0 running, 1 done, 2 failed
// (code and message kept for the loop's thread, which joins it).
struct Lane {
  std::unique_ptr<Cohort> c;
  std::thread th;
  std::atomic<int> state{0};
  int code = FX_OK;
  std::string err;
};

struct Server {
  fx_engine* engine = nullptr;
  int device = 0;
  int64_t budget = 0;
  int max_cohort = 32;
  int max_lanes = 4;
  std::vector<Request> reqs;
  std::unordered_map<int64_t, size_t> by_id;
  bool ran = false;

  void start_cohort(std::deque<size_t>& pending, Cohort& c, int64_t& resident, bool others, double now) {
    const Request& head = reqs[pending.front()];
    std::vector<size_t> members;
    int64_t foot = 0;
    while (!pending.empty() && static_cast<int>(members.size()) < max_cohort) {
      const Request& r = reqs[pending.front()];
      if (r.cycles != head.cycles || r.spc != head.spc || r.tol != head.tol || r.cg_rtol != head.cg_rtol ||
          r.max_newton != head.max_newton || r.cg_max_it != head.cg_max_it)
        break;
      if ((others || !members.empty()) && resident + foot + r.footprint > budget) break;
      members.push_back(pending.front());
      foot += r.footprint;
      pending.pop_front();
    }
    if (members.empty()) return;
    std::vector<fx_mesh> meshes;
    for (size_t i : members) meshes.push_back(reqs[i].mesh);
    fx_solve_opts o{};
    o.rtol = head.cg_rtol;
    o.atol = 0.0;
    o.max_iterations = head.cg_max_it;
    o.lanes = 32;
    FX_CUDA(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
    ck(fx_nbatch_create(meshes.data(), static_cast<int32_t>(meshes.size()), device, o, &c.nb), "fx_nbatch_create");
    const size_t m = members.size();
    c.offsets.assign(m + 1, 0);
    c.neq.assign(m, 0);
    ck(fx_nbatch_layout(c.nb, c.offsets.data(), c.neq.data()), "fx_nbatch_layout");
    const int64_t total = c.offsets[m];
    std::vector<double> F(static_cast<size_t>(total), 0.0);
    std::vector<int64_t> idx(m);
    for (size_t i = 0; i < m; ++i) {
      const Request& r = reqs[members[i]];
      if (static_cast<int64_t>(r.unit.size()) != c.neq[i])
        throw Error(FX_E_INVALID, "fx_server: a J2 request's load has the wrong length");
      std::copy(r.unit.begin(), r.unit.end(), F.begin() + c.offsets[i]);
      idx[i] = c.offsets[i] + r.monitor;
    }
    c.factors = cyclic_factors(head.cycles, head.spc);
    c.F.upload(F);
    c.fext.alloc(static_cast<size_t>(total));
    c.u.alloc(static_cast<size_t>(total));
    c.u.zero(c.st);
    c.idx.upload(idx);
    c.hist.alloc(c.factors.size() * m);
    c.members = members;
    c.conv.assign(m, 1);
    c.newton.assign(m, {});
    c.k = 0;
    c.footprint = foot;
    resident += foot;
    for (size_t i : members) reqs[i].admitted = now;
  }

  // one load step of the cohort; true when its path has ended (the members' results are kept)
  bool step_cohort(Cohort& c, double& now_out, const std::function<double()>& now) {
    const size_t m = c.members.size();
    const int64_t total = c.offsets[m];
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 4096)));
    k_scaled<<<grid, 256, 0, c.st>>>(c.F.ptr, c.factors[c.k], c.fext.ptr, total);
    FX_LAUNCH_CHECK("server_load");
    std::vector<int32_t> it(m);
    std::vector<fx_solve_result> res(m);
    const Request& head = reqs[c.members[0]];
    ck(fx_nbatch_step(c.nb, c.fext.ptr, c.u.ptr, head.tol, head.max_newton, it.data(), res.data(), c.st),
       "fx_nbatch_step");
    ck(fx_force_commit(fx_nbatch_force(c.nb), c.st), "fx_force_commit");
    k_pick<<<static_cast<unsigned>((m + 127) / 128), 128, 0, c.st>>>(c.u.ptr, c.idx.ptr, static_cast<int>(m),
                                                                   c.hist.ptr + static_cast<size_t>(c.k) * m);
    FX_LAUNCH_CHECK("server_monitor");
    for (size_t i = 0; i < m; ++i) {
      c.conv[i] = c.conv[i] && res[i].converged;
      c.newton[i].push_back(it[i]);
    }
    if (++c.k < static_cast<int>(c.factors.size())) return false;
    std::vector<double> u(static_cast<size_t>(total)), hist(c.hist.n);
    FX_CUDA(cudaMemcpyAsync(u.data(), c.u.ptr, sizeof(double) * u.size(), cudaMemcpyDeviceToHost, c.st));
    FX_CUDA(cudaMemcpyAsync(hist.data(), c.hist.ptr, sizeof(double) * hist.size(), cudaMemcpyDeviceToHost, c.st));
    FX_CUDA(cudaStreamSynchronize(c.st));
    now_out = now();
    for (size_t i = 0; i < m; ++i) {
      Request& r = reqs[c.members[i]];
      r.x.assign(u.begin() + c.offsets[i], u.begin() + c.offsets[i] + c.neq[i]);
      r.n = c.neq[i];
      r.hist.resize(c.factors.size());
      for (size_t s = 0; s < c.factors.size(); ++s) r.hist[s] = hist[s * m + i];
      r.newton = c.newton[i];
      r.res = fx_solve_result{};
      r.res.converged = c.conv[i];
      r.res.status = c.conv[i] ? FX_OK : FX_E_DIVERGED;
      r.done = now_out;
    }
    return true;
  }

  // a lane's thread: the cohort's load steps until its path ends or the loop stops
  void lane_main(Lane& L, const std::atomic<bool>& stop, const std::function<double()>& now) {
    try {
      FX_CUDA(cudaSetDevice(device));
      double done_at = 0.0;
      while (!stop.load(std::memory_order_relaxed) && !step_cohort(*L.c, done_at, now)) {
      }
      L.c->release();
      L.state.store(1);
    } catch (const Error& e) {
      L.code = e.code;
      L.err = e.what();
      L.state.store(2);
    } catch (const std::exception& e) {
      L.code = FX_E_INVALID;
      L.err = e.what();
      L.state.store(2);
    }
  }

  double run(bool realtime) {
    // the clock, the lanes and the stop flag outlive every lane thread (joined here on an error)
    using clock = std::chrono::steady_clock;
    const auto t0 = clock::now();
    const std::function<double()> now = [t0]() { return std::chrono::duration<double>(clock::now() - t0).count(); };
    std::vector<std::unique_ptr<Lane>> lanes;
    std::atomic<bool> stop{false};
    try {
      const double t = serve(realtime, now, lanes, stop);
      ran = true;
      return t;
    } catch (...) {
      stop.store(true);
      for (auto& L : lanes)
        if (L->th.joinable()) L->th.join();
      throw;
    }
  }

  double serve(bool realtime, const std::function<double()>& now, std::vector<std::unique_ptr<Lane>>& lanes,
               std::atomic<bool>& stop) {
    FX_CUDA(cudaSetDevice(device));
    std::vector<size_t> order(reqs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return reqs[a].arrival < reqs[b].arrival; });
    std::deque<size_t> pending, pending_j2;
    std::map<int32_t, size_t> slots;
    int64_t resident = 0;
    size_t nxt = 0;
    while (nxt < order.size() || !pending.empty() || !pending_j2.empty() || !slots.empty() || !lanes.empty()) {
      const double t = realtime ? now() : INFINITY;
      while (nxt < order.size() && reqs[order[nxt]].arrival <= t) {
        const size_t i = order[nxt++];
        (reqs[i].kind == 1 ? pending_j2 : pending).push_back(i);
      }
      // admissions in arrival order, while the footprint fits and the engine has room
      while (!pending.empty()) {
        Request& r = reqs[pending.front()];
        if ((!slots.empty() || !lanes.empty()) && resident + r.footprint > budget) break;
        int32_t slot = -1;
        const int rc = fx_engine_admit(engine, r.f, r.b.data(), &slot);
        if (rc == FX_E_NOMEM) break;
        ck(rc, "fx_engine_admit");
        slots[slot] = pending.front();
        pending.pop_front();
        resident += r.footprint;
        r.admitted = now();
      }
      if (slots.empty() && lanes.empty() && !pending.empty())
        throw Error(FX_E_NOMEM, "fx_server: request " + std::to_string(reqs[pending.front()].id) +
                                    " does not fit the engine even alone");
      // lanes whose path has ended: joined, their footprint released
      for (auto it = lanes.begin(); it != lanes.end();) {
        Lane& L = **it;
        const int st = L.state.load();
        if (st == 0) {
          ++it;
          continue;
        }
        L.th.join();
        if (st == 2) throw Error(L.code, L.err);
        resident -= L.c->footprint;
        it = lanes.erase(it);
      }
      while (static_cast<int>(lanes.size()) < max_lanes && !pending_j2.empty()) {
        auto L = std::make_unique<Lane>();
        L->c = std::make_unique<Cohort>();
        start_cohort(pending_j2, *L->c, resident, !slots.empty() || !lanes.empty(), now());
        if (L->c->members.empty()) {
          if (slots.empty() && lanes.empty())
            throw Error(FX_E_NOMEM, "fx_server: J2 request " + std::to_string(reqs[pending_j2.front()].id) +
                                        " does not fit the budget even alone");
          break;
        }
        Lane* lp = L.get();
        lanes.push_back(std::move(L));
        lp->th = std::thread([this, lp, &stop, &now]() { lane_main(*lp, stop, now); });
      }
      if (slots.empty()) {
        // nothing for this thread to advance: wait for an arrival or a lane's end
        double wait = lanes.empty() ? 0.01 : kPoll;
        if (nxt < order.size() && realtime) wait = std::min(wait, reqs[order[nxt]].arrival - now());
        else if (lanes.empty()) continue;
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
        continue;
      }
      // one engine tick (8 inner iterations; admissions and arrivals are looked at between ticks)
      int32_t running = 0;
      ck(fx_engine_round(engine, &running), "fx_engine_round");
      for (auto it = slots.begin(); it != slots.end();) {
        int32_t fin = 0;
        ck(fx_engine_finished(engine, it->first, &fin), "fx_engine_finished");
        if (!fin) {
          ++it;
          continue;
        }
        Request& r = reqs[it->second];
        r.x.assign(static_cast<size_t>(r.n), 0.0);
        ck(fx_engine_retire(engine, it->first, r.x.data(), &r.res), "fx_engine_retire");
        r.done = now();
        resident -= r.footprint;
        it = slots.erase(it);
      }
    }
    return now();
  }
};

}  // namespace
}  // namespace fx

struct fx_server {
  fx::Server s;
};

extern "C" {

int fx_server_create(fx_engine* engine, int32_t device, int64_t hbm_budget, int32_t max_cohort, int32_t max_lanes,
                     fx_server** out) {
  return fx::guard([&] {
    if (!engine || !out || hbm_budget < 0 || max_cohort <= 0 || max_lanes <= 0)
      throw fx::Error(FX_E_INVALID, "fx_server_create: bad arguments");
    auto* h = new fx_server;
    h->s.engine = engine;
    h->s.device = device;
    h->s.budget = hbm_budget;
    h->s.max_cohort = max_cohort;
    h->s.max_lanes = max_lanes;
    *out = h;
  });
}

void fx_server_destroy(fx_server* s) { delete s; }

int fx_server_add_static(fx_server* s, int64_t id, fx_force* f, const double* b_host, double arrival) {
  return fx::guard([&] {
    if (!s || !f || !b_host || !(arrival >= 0.0)) throw fx::Error(FX_E_INVALID, "fx_server_add_static: bad arguments");
    if (s->s.by_id.count(id)) throw fx::Error(FX_E_INVALID, "fx_server_add_static: the id is taken");
    int64_t info[9];
    fx::ck(fx_force_info(f, info), "fx_force_info");
    fx::Request r;
    r.id = id;
    r.kind = 0;
    r.arrival = arrival;
    r.f = f;
    r.n = info[0];
    r.b.assign(b_host, b_host + r.n);
    r.footprint = info[7];
    s->s.by_id[id] = s->s.reqs.size();
    s->s.reqs.push_back(std::move(r));
  });
}

int fx_server_add_j2(fx_server* s, int64_t id, const fx_mesh* mesh, const double* unit_load, int64_t monitor,
                     int32_t cycles, int32_t steps_per_cycle, double tol, int32_t max_newton, double cg_rtol,
                     int32_t cg_max_iterations, double arrival) {
  return fx::guard([&] {
    if (!s || !mesh || !unit_load || cycles <= 0 || steps_per_cycle <= 0 || !(tol > 0) || max_newton <= 0 ||
        !(cg_rtol > 0) || cg_max_iterations <= 0 || !(arrival >= 0.0) || monitor < 0 ||
        monitor >= mesh->num_equations)
      throw fx::Error(FX_E_INVALID, "fx_server_add_j2: bad arguments");
    if (s->s.by_id.count(id)) throw fx::Error(FX_E_INVALID, "fx_server_add_j2: the id is taken");
    fx::Request r;
    r.id = id;
    r.kind = 1;
    r.arrival = arrival;
    r.mesh = *mesh;
    r.unit.assign(unit_load, unit_load + mesh->num_equations);
    r.monitor = monitor;
    r.cycles = cycles;
    r.spc = steps_per_cycle;
    r.tol = tol;
    r.max_newton = max_newton;
    r.cg_rtol = cg_rtol;
    r.cg_max_it = cg_max_iterations;
    r.n = mesh->num_equations;
    r.footprint = fx::j2_footprint(*mesh);
    s->s.by_id[id] = s->s.reqs.size();
    s->s.reqs.push_back(std::move(r));
  });
}

int fx_server_run(fx_server* s, int32_t realtime, double* wall_seconds) {
  return fx::guard([&] {
    if (!s) throw fx::Error(FX_E_INVALID, "fx_server_run: null handle");
    if (s->s.ran) throw fx::Error(FX_E_INVALID, "fx_server_run: a server runs its requests once");
    const double w = s->s.run(realtime != 0);
    if (wall_seconds) *wall_seconds = w;
  });
}

int fx_server_result(const fx_server* s, int64_t id, double* x_host, fx_solve_result* r, double* times,
                     double* monitor, int32_t* newton) {
  return fx::guard([&] {
    if (!s) throw fx::Error(FX_E_INVALID, "fx_server_result: null handle");
    auto it = s->s.by_id.find(id);
    if (it == s->s.by_id.end()) throw fx::Error(FX_E_INVALID, "fx_server_result: no such request");
    const fx::Request& q = s->s.reqs[it->second];
    if (q.done < 0) throw fx::Error(FX_E_INVALID, "fx_server_result: the request has not been served");
    if (x_host) std::copy(q.x.begin(), q.x.end(), x_host);
    if (r) *r = q.res;
    if (times) {
      times[0] = q.arrival;
      times[1] = q.admitted;
      times[2] = q.done;
    }
    if (monitor) std::copy(q.hist.begin(), q.hist.end(), monitor);
    if (newton) std::copy(q.newton.begin(), q.newton.end(), newton);
  });
}

}  // extern "C"
