// sweep.cpp -- batched lumped-port sweep over many independent grids.
//
// Each instance gets its own engine (and with it its own CUDA stream and
// graphs); `concurrency` host worker threads take instances from a shared
// counter and drive one engine each, so the kernels of several small grids
// run side by side on the device.  Per instance: the port resistor is folded
// into the edge's Ca/Cb (oems_operator_set_lumped), the source voltage is a
// soft source scaled by the returned factor, the port voltage / current are
// f64 probes with running DFTs, and batches run until the energy has decayed
// by the requested dB below its peak (the peak carried across batches) or the
// step cap.  S11 follows Port.CalcPort (python/openEMS/ports.py:136-138).
// oems_sweep_run_until stops every instance at a step count and keeps its
// engine: a later call continues it where it stopped (the same bits as an
// uninterrupted run), oems_sweep_finish ends it with its partial DFTs.
// With packing on (oems_sweep_set_packed), run / run_until step the
// instances that are at the same step count together through one pack
// (oems_pack_run_batch): shared launches over all their grids instead of one
// stream per instance, with the same bits per instance.
// Only the public C ABI of the engine and the host operator is used.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/oems.h"
#include "../../include/oems_host.h"

namespace oems {
extern thread_local std::string g_last_error;
}

namespace {

struct Instance {
  oems_operator* op = nullptr;
  oems_sweep_instance desc{};
  bool done = false;  // ended: decayed, at max_timesteps, finished by the caller or failed
  oems_sweep_result res{};
  std::string error;
  std::vector<double> uf, if_;
  std::vector<double> trace;  // [step][2]: u, i (first trace_steps steps)
  // state of a started instance, kept between calls while it is paused
  oems_engine* en = nullptr;
  oems_excitation wave{};
  double dt = 0.0, peak = 0.0;
  uint64_t run = 0;
  int32_t du = -1, di = -1;
};

oems_status sfail(oems_status st, const char* msg) {
  oems::g_last_error = msg;
  return st;
}

}  // namespace

struct oems_sweep {
  int32_t device = -1;
  uint32_t concurrency = 1;
  uint32_t flags = 0;
  std::vector<double> freqs;
  std::vector<std::unique_ptr<Instance>> inst;
  double wall = 0.0, cell_steps = 0.0;
  uint64_t trace_steps = 0;
  bool packed = false;
};

namespace {

// Probe of one port quantity with the weights negated: u = +E . dl and the
// current delivered into the structure (oems_probe_port_terms gives -E . dl
// and the loop integral of H).
oems_status port_probe(oems_engine* en, const oems_operator* op, const uint64_t pos[3], int32_t dir, int32_t kind,
                       int32_t* id) {
  uint64_t n = 0;
  oems_status st = oems_probe_port_terms(op, pos, dir, kind, nullptr, 0, &n);
  if (st != OEMS_OK) return st;
  std::vector<oems_probe_term> t(std::max<uint64_t>(n, 1));
  st = oems_probe_port_terms(op, pos, dir, kind, t.data(), n, &n);
  if (st != OEMS_OK) return st;
  for (uint64_t k = 0; k < n; ++k) t[k].weight = -t[k].weight;
  return oems_engine_add_probe(en, t.data(), n, OEMS_PROBE_SUM_F64, id);
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Engine, CPML, port probes and DFTs of an instance (its operator is
// released once the engine holds the coefficients).
oems_status start_instance(const oems_sweep* sw, Instance& I) {
  const oems_sweep_instance& d = I.desc;
  double scale = 0.0;
  oems_status st = oems_operator_set_lumped(I.op, d.port_position, d.port_direction, d.port_resistance, 0.0,
                                            d.port_eps_r, d.port_sigma, &scale);
  if (st != OEMS_OK) return st;
  uint64_t dims[3];
  double delta[3];
  oems_operator_info(I.op, dims, &I.dt, delta);
  I.res.cells = (double)dims[0] * (double)dims[1] * (double)dims[2];
  oems_operator_desc od;
  st = oems_operator_engine_desc(I.op, sw->device, sw->flags, &od);
  if (st != OEMS_OK) return st;
  if ((st = oems_engine_create(&od, &I.en)) != OEMS_OK) return st;
  bool cpml = false;
  for (int f = 0; f < 6; ++f) cpml = cpml || d.cpml.layers[f] > 0;
  if (cpml && (st = oems_engine_add_cpml(I.en, &d.cpml)) != OEMS_OK) return st;
  int32_t pu = -1, pi = -1;
  if ((st = port_probe(I.en, I.op, d.port_position, d.port_direction, 0, &pu)) != OEMS_OK) return st;
  if ((st = port_probe(I.en, I.op, d.port_position, d.port_direction, 1, &pi)) != OEMS_OK) return st;
  const uint64_t nf = sw->freqs.size();
  if ((st = oems_engine_add_probe_dft(I.en, pu, sw->freqs.data(), nf, &I.du)) != OEMS_OK) return st;
  if ((st = oems_engine_add_probe_dft(I.en, pi, sw->freqs.data(), nf, &I.di)) != OEMS_OK) return st;
  // the engine holds its own copy of the coefficients from here on
  oems_operator_destroy(I.op);
  I.op = nullptr;
  I.wave = d.waveform;
  I.wave.amplitude *= scale;
  return OEMS_OK;
}

void end_instance(Instance& I) {
  if (I.en) oems_engine_destroy(I.en);
  I.en = nullptr;
  I.done = true;
  I.res.paused = 0;
}

// One batch of an instance: n steps from its current step, with the port
// source's samples, energy samples and decay checks every 100 steps and the
// peak carried in.
struct BatchBuf {
  std::vector<float> samples;
  std::vector<oems_energy_sample> es;
  oems_scheduled_excitation x{};
  oems_batch b{};
  oems_batch_result r{};
};

oems_status prepare_batch(const Instance& I, uint64_t n, BatchBuf& B) {
  const oems_sweep_instance& d = I.desc;
  B.samples.resize(std::max<uint64_t>(n, 1));
  B.es.resize(n / 100 + 2);
  const oems_status st = oems_excitation_sample(&I.wave, I.run, n, I.dt, B.samples.data());
  if (st != OEMS_OK) return st;
  B.x = oems_scheduled_excitation{};
  for (int a = 0; a < 3; ++a) B.x.position[a] = d.port_position[a];
  B.x.direction = (uint32_t)d.port_direction;
  B.x.soft_source = 1;
  B.x.samples = B.samples.data();
  B.x.num_samples = n;
  B.b = oems_batch{};
  B.b.num_steps = n;
  B.b.excitations = &B.x;
  B.b.num_excitations = 1;
  B.b.has_energy_decay_db = d.energy_decay_db != 0.0 ? 1 : 0;
  B.b.energy_decay_db = std::fabs(d.energy_decay_db);
  B.b.check_interval = 100;
  B.b.sample_interval = 100;
  B.b.track_peak = 1;
  B.b.initial_peak_energy = I.peak;
  B.r = oems_batch_result{};
  B.r.energy_samples = B.es.data();
  B.r.energy_capacity = B.es.size();
  return OEMS_OK;
}

// Folds a finished batch into the instance: traces, counters, peak and
// termination; `ended` is set when the batch ended the instance.
oems_status apply_batch(const oems_sweep* sw, Instance& I, BatchBuf& B, bool& ended) {
  const oems_batch_result& r = B.r;
  const std::vector<oems_energy_sample>& es = B.es;
  oems_status st = OEMS_OK;
  {
    if (sw->trace_steps > I.run) {
      // port u / i of this batch, kept up to trace_steps
      const uint64_t keep = std::min<uint64_t>(r.timesteps_executed, sw->trace_steps - I.run);
      std::vector<double> tr(2 * std::max<uint64_t>(r.timesteps_executed, 1));
      uint64_t got = 0;
      if ((st = oems_engine_read_probe_traces(I.en, tr.data(), r.timesteps_executed, &got)) != OEMS_OK) return st;
      I.trace.insert(I.trace.end(), tr.begin(), tr.begin() + 2 * std::min(keep, got));
    }
    uint64_t launches = 0;
    double dev_s = 0.0;
    oems_engine_last_batch_stats(I.en, &launches, &dev_s);
    I.res.device_seconds += dev_s;
    I.run += r.timesteps_executed;
    I.peak = std::max(I.peak, r.peak_energy);
    I.res.termination_reason = r.termination_reason;
    const uint64_t ns = std::min<uint64_t>(r.num_energy_samples, es.size());
    if (r.termination_reason == OEMS_TERMINATION_ENERGY_DECAY)
      I.res.final_decay_db = r.final_decay_db;
    else if (ns > 0 && I.peak > 0.0 && es[ns - 1].total_energy > 0.0)
      I.res.final_decay_db = 10.0 * std::log10(es[ns - 1].total_energy / I.peak);
    if (r.termination_reason != OEMS_TERMINATION_STEPS_COMPLETED || r.timesteps_executed == 0) ended = true;
  }
  return OEMS_OK;
}

// After the last batch of a call: reads the port DFTs back, then ends the
// instance or leaves it paused.
oems_status close_advance(const oems_sweep* sw, Instance& I, bool ended) {
  const uint64_t nf = sw->freqs.size();
  oems_status st = OEMS_OK;
  ended = ended || I.run >= I.desc.max_timesteps;
  I.res.timesteps = I.run;
  I.uf.assign(2 * nf, 0.0);
  I.if_.assign(2 * nf, 0.0);
  if ((st = oems_engine_read_probe_dft(I.en, I.du, I.uf.data())) != OEMS_OK) return st;
  if ((st = oems_engine_read_probe_dft(I.en, I.di, I.if_.data())) != OEMS_OK) return st;
  if (ended)
    end_instance(I);
  else
    I.res.paused = 1;
  return OEMS_OK;
}

// Runs batches until the instance ends or has run `cap` steps in total; the
// port DFTs so far are read back either way.
oems_status advance(const oems_sweep* sw, Instance& I, uint64_t batch, uint64_t cap) {
  const uint64_t limit = std::min<uint64_t>(cap, I.desc.max_timesteps);
  BatchBuf B;
  oems_status st = OEMS_OK;
  bool ended = I.run >= I.desc.max_timesteps;
  while (!ended && I.run < limit) {
    if ((st = prepare_batch(I, std::min(limit - I.run, batch), B)) != OEMS_OK) return st;
    if ((st = oems_engine_run_batch(I.en, &B.b, &B.r)) != OEMS_OK) return st;
    if ((st = apply_batch(sw, I, B, ended)) != OEMS_OK) return st;
  }
  return close_advance(sw, I, ended);
}

oems_status run_instance(const oems_sweep* sw, Instance& I, uint64_t batch, uint64_t cap) {
  if (!I.en) {
    const auto t_start = std::chrono::steady_clock::now();
    const oems_status st = start_instance(sw, I);
    I.res.setup_seconds = seconds_since(t_start);
    if (st != OEMS_OK) return st;
  }
  return advance(sw, I, batch, cap);
}

// Packed run: starts every instance (set-up on `concurrency` threads), then
// steps the instances that are at the same step count together through one
// pack, batch by batch, each batch as long as the shortest remaining run of
// the group allows (the results do not depend on batch boundaries).  An
// instance leaves the group when it ends or reaches its cap; groups are
// formed until every instance has ended or stopped at its cap.
oems_status run_packed(oems_sweep* s, std::vector<Instance*>& todo, uint64_t batch, uint64_t cap) {
  std::atomic<size_t> next{0};
  auto starter = [&]() {
    for (size_t k = next++; k < todo.size(); k = next++) {
      Instance& I = *todo[k];
      if (I.en) continue;
      const auto t_start = std::chrono::steady_clock::now();
      const oems_status st = start_instance(s, I);
      I.res.setup_seconds = seconds_since(t_start);
      I.res.status = st;
      if (st != OEMS_OK) {
        I.error = oems_last_error_message();
        end_instance(I);
      }
    }
  };
  {
    const size_t nthreads = std::min<size_t>(s->concurrency, todo.size());
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nthreads; ++t) pool.emplace_back(starter);
    if (nthreads > 0) starter();
    for (auto& t : pool) t.join();
  }
  auto limit_of = [&](const Instance& I) { return std::min<uint64_t>(cap, I.desc.max_timesteps); };
  auto fail_instance = [&](Instance& I, oems_status st) {
    I.res.status = st;
    I.error = oems_last_error_message();
    end_instance(I);
  };
  while (true) {
    // the next group: live instances below their cap at the smallest step count
    std::vector<Instance*> live;
    for (Instance* I : todo)
      if (!I->done && I->en && I->res.status == OEMS_OK) live.push_back(I);
    std::vector<Instance*> group;
    uint64_t r0 = UINT64_MAX;
    for (Instance* I : live)
      if (I->run < limit_of(*I) && I->run < I->desc.max_timesteps) r0 = std::min(r0, I->run);
    for (Instance* I : live)
      if (I->run == r0 && I->run < limit_of(*I) && I->run < I->desc.max_timesteps) group.push_back(I);
    if (group.empty()) break;
    std::vector<oems_engine*> engines;
    for (Instance* I : group) engines.push_back(I->en);
    oems_pack* pack = nullptr;
    oems_status st = oems_pack_create(engines.data(), engines.size(), &pack);
    if (st != OEMS_OK) return st;
    const auto t_group = std::chrono::steady_clock::now();
    std::vector<BatchBuf> bufs(group.size());
    std::vector<char> in(group.size(), 1), ended(group.size(), 0);
    std::vector<const oems_batch*> bp(group.size(), nullptr);
    std::vector<oems_batch_result> res(group.size());
    std::vector<oems_status> sts(group.size(), OEMS_OK);
    size_t left = group.size();
    while (left > 0) {
      uint64_t n = batch;
      for (size_t k = 0; k < group.size(); ++k)
        if (in[k]) n = std::min(n, limit_of(*group[k]) - group[k]->run);
      for (size_t k = 0; k < group.size(); ++k) {
        bp[k] = nullptr;
        if (!in[k]) continue;
        if ((st = prepare_batch(*group[k], n, bufs[k])) != OEMS_OK) {
          oems_pack_destroy(pack);
          return st;
        }
        bp[k] = &bufs[k].b;
        res[k] = bufs[k].r;  // energy sample buffer and capacity
      }
      if ((st = oems_pack_run_batch(pack, bp.data(), res.data(), sts.data())) != OEMS_OK) {
        oems_pack_destroy(pack);
        return st;
      }
      for (size_t k = 0; k < group.size(); ++k) {
        if (!in[k]) continue;
        Instance& I = *group[k];
        bufs[k].r = res[k];
        bool e = false;
        if (sts[k] != OEMS_OK) {
          oems::g_last_error = "field energy became NaN or infinite";
          fail_instance(I, sts[k]);
          in[k] = 0;
          --left;
          continue;
        }
        if ((st = apply_batch(s, I, bufs[k], e)) != OEMS_OK) {
          fail_instance(I, st);
          in[k] = 0;
          --left;
          continue;
        }
        if (e || I.run >= limit_of(I) || I.run >= I.desc.max_timesteps) {
          ended[k] = e ? 1 : 0;
          in[k] = 0;
          --left;
        }
      }
    }
    oems_pack_destroy(pack);
    const double group_s = seconds_since(t_group);
    for (size_t k = 0; k < group.size(); ++k) {
      Instance& I = *group[k];
      I.res.host_seconds += group_s;
      if (I.done) continue;  // failed above
      if ((st = close_advance(s, I, ended[k] != 0)) != OEMS_OK) fail_instance(I, st);
    }
  }
  return OEMS_OK;
}

}  // namespace

extern "C" {

oems_status oems_sweep_set_packed(oems_sweep* s, int32_t on) {
  if (!s) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL sweep");
  s->packed = on != 0;
  return OEMS_OK;
}

oems_status oems_sweep_create(int32_t device, uint32_t concurrency, uint32_t engine_flags, const double* freqs,
                              uint64_t nfreq, oems_sweep** out) {
  if (!out || (!freqs && nfreq)) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (nfreq == 0) return sfail(OEMS_ERR_CONFIG, "a sweep needs at least one frequency");
  if (concurrency == 0) return sfail(OEMS_ERR_CONFIG, "concurrency must be at least 1");
  auto* s = new oems_sweep;
  s->device = device;
  s->concurrency = concurrency;
  s->flags = engine_flags;
  s->freqs.assign(freqs, freqs + nfreq);
  *out = s;
  return OEMS_OK;
}

void oems_sweep_destroy(oems_sweep* s) {
  if (!s) return;
  for (auto& I : s->inst) {
    if (I->en) oems_engine_destroy(I->en);
    oems_operator_destroy(I->op);
  }
  delete s;
}

oems_status oems_sweep_add(oems_sweep* s, const oems_sweep_instance* d, int32_t* id) {
  if (!s || !d || !d->op) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  uint64_t dims[3];
  double dt, delta[3];
  oems_operator_info(d->op, dims, &dt, delta);
  if (d->port_direction < 0 || d->port_direction > 2) return sfail(OEMS_ERR_CONFIG, "port direction must be 0..2");
  for (int a = 0; a < 3; ++a)
    if (d->port_position[a] >= dims[a]) return sfail(OEMS_ERR_CONFIG, "port outside the grid");
  if (!(d->port_resistance > 0.0)) return sfail(OEMS_ERR_CONFIG, "port resistance must be positive");
  if (!(d->port_eps_r > 0.0) || d->port_sigma < 0.0) return sfail(OEMS_ERR_MATERIAL, "invalid port background");
  if (d->max_timesteps == 0) return sfail(OEMS_ERR_CONFIG, "max_timesteps must be positive");
  auto I = std::make_unique<Instance>();
  oems_status st = oems_operator_clone(d->op, &I->op);
  if (st != OEMS_OK) return st;
  I->desc = *d;
  I->desc.op = nullptr;
  s->inst.push_back(std::move(I));
  if (id) *id = (int32_t)s->inst.size() - 1;
  return OEMS_OK;
}

oems_status oems_sweep_run_until(oems_sweep* s, uint64_t batch_steps, uint64_t step_cap) {
  if (!s) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL sweep");
  const uint64_t batch = batch_steps ? batch_steps : 2000;
  std::vector<Instance*> todo;
  for (auto& I : s->inst)
    if (!I->done) todo.push_back(I.get());
  std::vector<uint64_t> before(todo.size());
  for (size_t k = 0; k < todo.size(); ++k) before[k] = todo[k]->run;
  if (s->packed) {
    const auto t0 = std::chrono::steady_clock::now();
    const oems_status st = run_packed(s, todo, batch, step_cap);
    s->wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    s->cell_steps = 0.0;
    for (size_t k = 0; k < todo.size(); ++k)
      s->cell_steps += todo[k]->res.cells * (double)(todo[k]->run - before[k]);
    if (st != OEMS_OK) return st;
    for (Instance* I : todo)
      if (I->res.status != OEMS_OK) {
        oems::g_last_error = "sweep instance failed: " + I->error;
        return (oems_status)I->res.status;
      }
    return OEMS_OK;
  }
  std::atomic<size_t> next{0};
  const auto t0 = std::chrono::steady_clock::now();
  auto worker = [&]() {
    for (size_t k = next++; k < todo.size(); k = next++) {
      Instance& I = *todo[k];
      const auto t_inst = std::chrono::steady_clock::now();
      const oems_status st = run_instance(s, I, batch, step_cap);
      I.res.status = st;
      if (st != OEMS_OK) {
        I.error = oems_last_error_message();
        end_instance(I);
      }
      I.res.host_seconds += seconds_since(t_inst);
    }
  };
  const size_t nthreads = std::min<size_t>(s->concurrency, todo.size());
  std::vector<std::thread> pool;
  for (size_t t = 1; t < nthreads; ++t) pool.emplace_back(worker);
  if (nthreads > 0) worker();
  for (auto& t : pool) t.join();
  s->wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  s->cell_steps = 0.0;
  for (size_t k = 0; k < todo.size(); ++k) s->cell_steps += todo[k]->res.cells * (double)(todo[k]->run - before[k]);
  for (Instance* I : todo)
    if (I->res.status != OEMS_OK) {
      oems::g_last_error = "sweep instance failed: " + I->error;
      return (oems_status)I->res.status;
    }
  return OEMS_OK;
}

oems_status oems_sweep_run(oems_sweep* s, uint64_t batch_steps) {
  return oems_sweep_run_until(s, batch_steps, UINT64_MAX);
}

oems_status oems_sweep_advance(oems_sweep* s, int32_t id, uint64_t batch_steps, uint64_t step_cap) {
  if (!s) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL sweep");
  if (id < 0 || id >= (int32_t)s->inst.size()) return sfail(OEMS_ERR_CONFIG, "unknown sweep instance");
  Instance& I = *s->inst[id];
  if (I.done) return OEMS_OK;
  const auto t_inst = std::chrono::steady_clock::now();
  const oems_status st = run_instance(s, I, batch_steps ? batch_steps : 2000, step_cap);
  I.res.status = st;
  if (st != OEMS_OK) {
    I.error = oems_last_error_message();
    end_instance(I);
  }
  I.res.host_seconds += seconds_since(t_inst);
  return st;
}

oems_status oems_sweep_finish(oems_sweep* s, int32_t id) {
  if (!s) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL sweep");
  if (id < 0 || id >= (int32_t)s->inst.size()) return sfail(OEMS_ERR_CONFIG, "unknown sweep instance");
  Instance& I = *s->inst[id];
  if (!I.done && !I.en) return sfail(OEMS_ERR_CONFIG, "sweep instance has not run");
  if (!I.done) end_instance(I);
  return OEMS_OK;
}

oems_status oems_sweep_get_result(const oems_sweep* s, int32_t id, oems_sweep_result* info, double* uf, double* if_,
                                  double* s11) {
  if (!s) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL sweep");
  if (id < 0 || id >= (int32_t)s->inst.size()) return sfail(OEMS_ERR_CONFIG, "unknown sweep instance");
  const Instance& I = *s->inst[id];
  if (info) *info = I.res;
  if (!I.done && !I.en) return sfail(OEMS_ERR_CONFIG, "sweep instance has not run");
  if (I.res.status != OEMS_OK) return sfail((oems_status)I.res.status, I.error.c_str());
  const size_t nf = s->freqs.size();
  if (uf) std::copy(I.uf.begin(), I.uf.end(), uf);
  if (if_) std::copy(I.if_.begin(), I.if_.end(), if_);
  if (s11) {
    const double R = I.desc.port_resistance;
    for (size_t f = 0; f < nf; ++f) {
      // u_inc = (u + i R) / 2, S11 = (u - u_inc) / u_inc
      const double ur = I.uf[2 * f], ui = I.uf[2 * f + 1];
      const double ir = I.if_[2 * f], ii = I.if_[2 * f + 1];
      const double ar = 0.5 * (ur + ir * R), ai = 0.5 * (ui + ii * R);
      const double br = ur - ar, bi = ui - ai;
      const double den = ar * ar + ai * ai;
      s11[2 * f] = den > 0.0 ? (br * ar + bi * ai) / den : 0.0;
      s11[2 * f + 1] = den > 0.0 ? (bi * ar - br * ai) / den : 0.0;
    }
  }
  return OEMS_OK;
}

oems_status oems_sweep_set_trace_steps(oems_sweep* s, uint64_t steps) {
  if (!s) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL sweep");
  s->trace_steps = steps;
  return OEMS_OK;
}

oems_status oems_sweep_get_trace(const oems_sweep* s, int32_t id, double* out, uint64_t cap_steps, uint64_t* nsteps) {
  if (!s) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL sweep");
  if (id < 0 || id >= (int32_t)s->inst.size()) return sfail(OEMS_ERR_CONFIG, "unknown sweep instance");
  const Instance& I = *s->inst[id];
  const uint64_t n = I.trace.size() / 2;
  if (nsteps) *nsteps = n;
  if (out) std::copy(I.trace.begin(), I.trace.begin() + 2 * std::min(n, cap_steps), out);
  return OEMS_OK;
}

oems_status oems_sweep_stats(const oems_sweep* s, double* wall, double* cell_steps) {
  if (!s) return sfail(OEMS_ERR_INVALID_ARGUMENT, "NULL sweep");
  if (wall) *wall = s->wall;
  if (cell_steps) *cell_steps = s->cell_steps;
  return OEMS_OK;
}

}  // extern "C"
