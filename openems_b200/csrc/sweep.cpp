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

// Runs batches until the instance ends or has run `cap` steps in total; the
// port DFTs so far are read back either way.
oems_status advance(const oems_sweep* sw, Instance& I, uint64_t batch, uint64_t cap) {
  const oems_sweep_instance& d = I.desc;
  const uint64_t nf = sw->freqs.size();
  const uint64_t limit = std::min<uint64_t>(cap, d.max_timesteps);
  std::vector<float> samples(batch);
  std::vector<oems_energy_sample> es(batch / 100 + 2);
  const bool has_decay = d.energy_decay_db != 0.0;
  oems_status st = OEMS_OK;
  bool ended = I.run >= d.max_timesteps;
  while (!ended && I.run < limit) {
    const uint64_t n = std::min(limit - I.run, batch);
    if ((st = oems_excitation_sample(&I.wave, I.run, n, I.dt, samples.data())) != OEMS_OK) return st;
    oems_scheduled_excitation x{};
    for (int a = 0; a < 3; ++a) x.position[a] = d.port_position[a];
    x.direction = (uint32_t)d.port_direction;
    x.soft_source = 1;
    x.samples = samples.data();
    x.num_samples = n;
    oems_batch b{};
    b.num_steps = n;
    b.excitations = &x;
    b.num_excitations = 1;
    b.has_energy_decay_db = has_decay ? 1 : 0;
    b.energy_decay_db = std::fabs(d.energy_decay_db);
    b.check_interval = 100;
    b.sample_interval = 100;
    b.track_peak = 1;
    b.initial_peak_energy = I.peak;
    oems_batch_result r{};
    r.energy_samples = es.data();
    r.energy_capacity = es.size();
    if ((st = oems_engine_run_batch(I.en, &b, &r)) != OEMS_OK) return st;
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
  ended = ended || I.run >= d.max_timesteps;
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

oems_status run_instance(const oems_sweep* sw, Instance& I, uint64_t batch, uint64_t cap) {
  if (!I.en) {
    const auto t_start = std::chrono::steady_clock::now();
    const oems_status st = start_instance(sw, I);
    I.res.setup_seconds = seconds_since(t_start);
    if (st != OEMS_OK) return st;
  }
  return advance(sw, I, batch, cap);
}

}  // namespace

extern "C" {

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
