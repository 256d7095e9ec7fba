"""Benchmark of the B200 engine for BSim's SGSim LIF step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--impl ours|reference]

A step is one simulation cycle (dt = 0.1 ms) of the whole network. The default
workload is the 1e6-neuron CUBA network (100 populations x 10,000 LIF_brian
neurons, ~1.19e9 synapses, ~500 Hz, delays U{1..6} steps), built on the device
by the seeded generator. Metric: synaptic events per second (one event = one
synapse delivering one spike), plus the realtime factor (simulated seconds per
wall second). With N > 1 (torchrun, one process per GPU) every rank simulates
its own replica (a different seed): the networks are independent, so there is
no data-path collective, only a barrier and a max over ranks of the timing.

--impl reference times the reference's own CPU simulator (oracle/_ref, built
from its sources) on a scaled-down replica of the same workload.
"""
import argparse
import json
import os
import signal
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 1.0e-4
HBM_FALLBACK_GBS = 6650.0
# Algorithmic bytes per unit of work of one step (the HBM roofline of the path):
BYTES_PER_NEURON_STEP = 52.0   # read/write v, i_E, i_I, refrac (32), v_tmp (4), read+clear E/I input (16)
BYTES_PER_EVENT = 8.0          # int32 target + fp32 weight of one delivered synapse
BYTES_PER_SPIKE = 8.0          # fired id written once, read once
# Delivery mode per workload when --delivery is not given: the fastest measured on
# a B200 (1e6-neuron network at ~545 Hz: tiled 0.223 ms per cycle, push ~0.44 ms).
# fastest measured delivery per workload (steady state): tiled on the 1e6-neuron network
# (-51 % against push); on the dense one tiled and push are level (2.95-3.11 ms against
# 3.03-3.08 ms per cycle over several boxes), and push varies less
DEFAULT_DELIVERY = {"plain_1m": "tile"}


def workload(name, seed):
    from bsim_b200 import workloads as W
    if name == "plain_1m":
        specs, _ = W.plain_1m(seed)
        desc = "100 x 10,000 LIF_brian CUBA, ~500 Hz, delays U{1..6}, p=0.1 chain + 20% remote"
    elif name == "plain_quarter":
        specs = [W.cuba(25, 10000, 500, 6, seed, i_max=30e-9)]
        desc = "25 x 10,000 LIF_brian CUBA, ~500 Hz, delays U{1..6} (profiling size: 2.4 GB of rows)"
    elif name == "standard_cpu":
        specs, _ = W.standard_cpu(seed)
        desc = "10 x 1,000 LIF_brian CUBA, ~100 Hz, delays U{1..6}"
    elif name == "dense_1m":
        specs, _ = W.dense_1m(seed)
        desc = "50 x 20,000 LIF_brian CUBA, ~2 kHz, delays U{1..50}"
    elif name == "dense_quarter":
        specs = [W.cuba(50, 5000, 2000, 50, seed, i_max=62.5e-9)]
        desc = "50 x 5,000 LIF_brian CUBA, ~2 kHz, delays U{1..50} (profiling size of the dense network)"
    elif name.startswith("batched"):
        k = int(name.split("_")[1]) if "_" in name else 256
        specs, _ = W.batched(k, seed)
        desc = "%d independent CUBA nets, populations U{5..40} x neurons U{500..8000}" % k
    else:
        raise SystemExit("unknown config " + name)
    return specs, desc


class ClockSampler:
    """Clocks, power and throttle reasons sampled while the timed steps run. A timed
    region of 20 cycles lasts a few milliseconds, so NVML is polled from the host between
    non-blocking queries of the region's end event (poll_until); where NVML cannot be
    loaded, nvidia-smi samples every 200 ms instead. Samples are kept as rows of
    nvidia-smi's csv fields (FIELDS) and summarised by summary()."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None
        self.nv = None
        self.rows = []

    def _nvml_handle(self):
        nv = self.nv
        try:
            import torch
            uuid = getattr(torch.cuda.get_device_properties(self.gpu), "uuid", None)
            if uuid is not None:
                return nv.nvmlDeviceGetHandleByUUID("GPU-" + str(uuid))
        except Exception:
            pass
        return nv.nvmlDeviceGetHandleByIndex(self.gpu)

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.handle = self._nvml_handle()
            self.sm_max = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.sample()  # the first queries take milliseconds: made before the region, not kept
            self.rows = []
            return self
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def sample(self):
        """One NVML sample (no-op without NVML)."""
        if not self.nv:
            return
        nv, h = self.nv, self.handle
        try:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
            rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            return
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        self.rows.append([str(self.gpu), str(sm), str(self.sm_max), "%.2f" % pw, "0x%x" % rs] +
                         ["Active" if rs & b else "Not Active" for b in bits])

    def poll_until(self, event, every_s=1e-4):
        """Samples (at most every `every_s`) until the CUDA event has completed, then waits for it."""
        self.sample()
        last = time.perf_counter()
        while not event.query():
            now = time.perf_counter()
            if now - last >= every_s:
                self.sample()
                last = now
        event.synchronize()

    def __exit__(self, *a):
        if self.nv:
            with open(self.path, "w") as f:
                for r in self.rows:
                    f.write(", ".join(r) + "\n")
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.send_signal(signal.SIGTERM)
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return float(json.load(open(p))["hbm_gbs"]), "measured"
        except (ValueError, KeyError):
            pass
    return HBM_FALLBACK_GBS, "fallback"


def profiled_traffic(config, delivery, alg_bytes):
    """DRAM bytes per launch of the step kernel: the committed ncu captures give
    DRAM bytes per algorithmic byte for a workload and delivery mode ("plain_1m/tile"),
    applied to this run's algorithmic bytes per launch. None if never captured."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        v = d.get("%s/%s" % (config, delivery))
        if isinstance(v, dict) and v.get("dram_bytes_per_alg_byte"):
            return v["dram_bytes_per_alg_byte"] * alg_bytes
    return None


def roofline_frac(neuron_steps, events, spikes, seconds):
    """Algorithmic bytes (52 B per neuron-step, 8 B per event, 8 B per spike) per second
    as a fraction of the measured HBM copy bandwidth."""
    peak, _ = measured_hbm_peak()
    alg = BYTES_PER_NEURON_STEP * neuron_steps + BYTES_PER_EVENT * events + BYTES_PER_SPIKE * spikes
    return alg / max(seconds, 1e-12) / 1e9 / peak


def reduce_over_ranks(dist, maxes, sums, device="cpu"):
    """Max over ranks of each value in `maxes` and sum over ranks of each value in
    `sums` (float64). With dist None (one process) the values come back unchanged.
    Every rank must call it with the same number of values."""
    import torch
    if dist is None:
        return [float(v) for v in maxes], [float(v) for v in sums]
    mx = torch.tensor([float(v) for v in maxes], dtype=torch.float64, device=device)
    sm = torch.tensor([float(v) for v in sums], dtype=torch.float64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx.tolist(), sm.tolist()


# ---------------------------------------------------------------------------
# CPU baselines (oracle/_ref: the reference's own simulator, else the oracle port)
# ---------------------------------------------------------------------------
def replica_net(spec, pop_size):
    """Scaled-down replica of a generated workload, in the reference API's terms. The
    generator is the oracle library's copy, so the CPU arms never load the engine."""
    from bsim_b200 import workloads as W
    from oracle import oracle
    rs = W.scaled(spec, pop_size)
    g = oracle.gen_host(rs)
    dt = np.float32(DT)
    net = dict(params=g["params"].astype(np.float64), pop_size=np.full(rs.n_pop, rs.pop_size, np.int64),
               pop_tau=np.tile([rs.tau_syn_E, rs.tau_syn_I], (rs.n_pop, 1)).astype(np.float64),
               src=g["src"], dst=g["dst"], weight=g["weight"].astype(np.float64),
               delay=(g["delay_steps"].astype(np.float32) * dt).astype(np.float64),
               type=(g["weight"] < 0).astype(np.uint8), dt=float(dt))
    return rs, g, net


def cpu_baseline(spec, steps, budget_s=20.0, copies=1):
    """Times the reference simulator (or the oracle port) on a replica sized so
    that the run takes about budget_s seconds. With copies > 1 that many reference
    processes run the replica at once (one per host CPU: the reference simulator is
    single-threaded, so its multi-core throughput is that of independent networks);
    events/s is the sum over copies over the slowest copy's loop time. Returns
    (events/s, dict)."""
    from oracle import oracle
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import netio
    S_full = spec.n_pop * (spec.pop_size ** 2) * spec.p_conn * 1.2
    ref = oracle.ref_available("f32")
    # the reference walks every synapse every step (~60 ns each on one core at these rates)
    pop = int(spec.pop_size * min(1.0, np.sqrt(budget_s / (60e-9 * S_full * steps))))
    # the reference holds ~90 B of host objects per synapse: all copies together stay
    # within 30 % of the available host memory (and 64 GB)
    avail = 64e9
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = min(avail, 0.3 * float(line.split()[1]) * 1024)
    except OSError:
        pass
    pop_mem = int(spec.pop_size * np.sqrt(avail / (copies * 90.0 * S_full)))
    pop = max(min(pop, pop_mem), 20)
    rs, g, net = replica_net(spec, pop)
    orc = oracle.run(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], np.float32(DT), steps)
    events = int(orc["events_per_step"].sum())
    if ref and copies > 1:
        with tempfile.TemporaryDirectory() as d:
            netio.write_net(os.path.join(d, "net.bin"), net, steps, 0)
            secs_all = oracle.run_reference_many(os.path.join(d, "net.bin"), copies, "f32")
        secs, kind = max(secs_all), "reference"
        events *= copies
    elif ref:
        copies = 1
        with tempfile.TemporaryDirectory() as d:
            netio.write_net(os.path.join(d, "net.bin"), net, steps, 0)
            r = oracle.run_reference(os.path.join(d, "net.bin"), os.path.join(d, "out.bin"), "f32",
                                     record=False, n=g["params"].shape[0], n_rec=0)
        secs, kind = r["seconds"], "reference"
    else:
        copies = 1
        t0 = time.perf_counter()
        oracle.run(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], np.float32(DT), steps)
        secs, kind = time.perf_counter() - t0, "port"
    sample = ("%s: %d steps of a %d x %d replica (%d synapses) of the same generator; %d %s; "
              "a replica of the same rates and out-degrees; smaller replicas fit the CPU caches better, so "
              "this is an upper bound on the full-size network's rate" %
              ("reference STSim float build (oracle/_ref)" if kind == "reference" else "oracle port",
               steps, rs.n_pop, rs.pop_size, len(g["src"]), copies,
               "thread" if copies == 1 else "single-threaded processes at once, one per host CPU"))
    return events / secs, dict(kind=kind, sample=sample, seconds=secs, events=events, copies=copies,
                               rtf=steps * DT / secs, replica_synapses=int(len(g["src"])))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    specs, desc = workload(args.config, 1)
    total = args.steps + args.warmup
    try:
        eps, info = cpu_baseline(specs[0], total, budget_s=60.0, copies=len(os.sched_getaffinity(0)))
    except Exception as ex:  # reference missing or failed
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU run failed: %s" % ex}))
        return
    line = {"impl": "reference", "metric": "synaptic events/s", "value": eps, "unit": "events/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * info["seconds"] / total, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": {"workload": args.config + ": " + desc, "sample": info["sample"]},
            "realtime_factor": info["rtf"],
            "cpu_baseline": {"value": eps, "unit": "events/s", "cores": info["copies"], "kind": info["kind"],
                             "sample": info["sample"]},
            "e2e": {"value": eps, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Batched + predictor-scheduled vs plain
# ---------------------------------------------------------------------------
def batched_vs_plain(n_nets, steps, device, warm=300):
    """The networks of the batched generator (populations U{5..40} x neurons
    U{500..8000}, 100/500/2000 Hz, delays U{1..6} or U{1..50}) run
    (a) plain: one engine per network, one after the other, each with the faster of
        push and tiled delivery (both are run; the better time is kept);
    (b) batched: all networks packed into one engine stepped by one launch per cycle
        (CUDA graphs of 100 cycles); each tile scans its own network's delay range.
        When the push rows fit beside the tiled copy the engine delivers AUTO under the
        exact schedule (cost models from the autotuner on the delivered window's spike
        count); otherwise it holds the tiled copy alone and delivers tiled.
    Same cycles, same dynamics: every network's spike counts are compared between (a)
    and (b)."""
    import torch
    import bsim_b200 as B
    from bsim_b200 import workloads as W
    specs, _ = W.batched(n_nets, seed=7)

    def timed(eng, k):
        st = torch.cuda.ExternalStream(eng.stream(), device=device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        i0 = eng.info().events_total
        e0.record(st)
        eng.run_async(k)
        e1.record(st)
        e1.synchronize()
        eng.sync()
        return e0.elapsed_time(e1), eng.info().events_total - i0

    import ctypes
    n_syn = 0
    for sp in specs:
        nn, ss = ctypes.c_int64(), ctypes.c_int64()
        B._check(B.lib().bsim_gen_count(ctypes.byref(sp), ctypes.byref(nn), ctypes.byref(ss)))
        n_syn += ss.value
    free, _ = torch.cuda.mem_get_info(device)
    # push rows (8 B per synapse) beside the tiled copy (~8.4 B per synapse plus offsets)
    schedule = "auto_exact" if 18.0 * n_syn < 0.85 * free else "tile"
    t_build = time.perf_counter()
    eb = B.Engine.generated(specs, DT, opts=B.options(device=device, graph_steps=100, delivery=(
        B.DELIVERY_AUTO if schedule == "auto_exact" else B.DELIVERY_TILE)))
    t_build = time.perf_counter() - t_build
    tune = None
    eb.run(warm)
    if schedule == "auto_exact":
        tune = eb.autotune(10)
        eb.set_predictor(None, cost_push=list(tune.cost_push), cost_tile=list(tune.cost_tile))
        # autotuning advanced the networks: the plain runs warm up to the same cycle
    warm_all = int(eb.info().steps_done)
    fc0 = eb.fire_count().astype(np.int64)
    ms_b, ev_b = timed(eb, steps)
    fc_b = eb.fire_count().astype(np.int64)
    spk_b = int((fc_b - fc0).sum())
    info = eb.info()
    st = eb.predictor_stats()
    eb.close()

    plain_ms, plain_ev, plain_spk, same = 0.0, 0, 0, True
    modes = {"push": 0, "tile": 0}
    base = 0
    for sp in specs:
        n = sp.n_pop * sp.pop_size
        best = None
        for name, dl in (("push", B.DELIVERY_PUSH), ("tile", B.DELIVERY_TILE)):
            e = B.Engine.generated(sp, DT, opts=B.options(device=device, graph_steps=100, delivery=dl))
            e.run(warm_all)
            c0 = e.fire_count().astype(np.int64)
            ms, ev = timed(e, steps)
            c1 = e.fire_count().astype(np.int64)
            e.close()
            same &= bool(np.array_equal(c1, fc_b[base:base + n]))
            if best is None or ms < best[1]:
                best = (name, ms, ev, int((c1 - c0).sum()))
        modes[best[0]] += 1
        plain_ms += best[1]
        plain_ev += best[2]
        plain_spk += best[3]
        base += n
    n_all = int(info.n_neurons)
    plain = plain_ev / (plain_ms / 1e3)
    batched = ev_b / (ms_b / 1e3)
    out = {"workload": "%d networks of the batched generator (seed 7), %d cycles each after %d warm-up cycles"
                       % (n_nets, steps, warm_all),
           "neurons": n_all, "synapses": int(info.n_synapses), "build_seconds": t_build,
           "plain_events_per_s": plain, "batched_events_per_s": batched, "ratio": batched / plain,
           "target_ratio": 3.0,
           "hbm_roofline_frac": {"plain": roofline_frac(n_all * steps, plain_ev, plain_spk, plain_ms / 1e3),
                                 "batched": roofline_frac(n_all * steps, ev_b, spk_b, ms_b / 1e3)},
           "plain_network_seconds_per_s": steps * DT * n_nets / (plain_ms / 1e3),
           "batched_network_seconds_per_s": steps * DT * n_nets / (ms_b / 1e3),
           "plain_best_modes": modes, "batched_engines": 1, "batched_schedule": schedule,
           "batched_timing": "CUDA events on the engine's stream", "spike_counts_identical": same}
    if tune is not None:
        out["autotune"] = {"delivery": tune.delivery, "block": tune.block_threads, "grid": tune.grid_blocks,
                           "cost_push_ns": list(tune.cost_push), "cost_tile_ns": list(tune.cost_tile)}
        out["schedule_stats"] = {"cycles": int(st.cycles), "tile_cycles": int(st.tile_cycles)}
    return out


def predicted_vs_plain(steps, device, settle=1000, chunk=50):
    """The predictor-scheduled workload (200 x 10,000 LIF_brian, delays U{1..20}, i_offset
    under a 10 Hz square wave) run three ways over the same cycles: plain push, plain
    tiled, and AUTO delivery chosen per cycle by the trained firing predictor with cost
    models fitted from the plain runs. Spike counts must agree; the report gives each
    mode's events/s, the predictor's count error and fallback rate."""
    import torch
    import bsim_b200 as B
    from bsim_b200 import predictor as PR
    from bsim_b200 import workloads as W
    specs, _ = W.predicted_2m(1)
    sp = specs[0]
    half = sp.drive_half_period

    t_train = time.perf_counter()
    counts, size, indeg = PR.collect(W.predicted_2m(2)[0], 3000, DT, settle=500, opts=B.options(device=device))
    x, y = PR.features(counts, size, indeg)
    params, loss = PR.train(x, y, epochs=3, batch=8192, lr=2e-3)
    t_train = time.perf_counter() - t_train

    def run_mode(deliv, setup=None):
        eng = B.Engine.generated(specs, DT, opts=B.options(device=device, delivery=deliv, graph_steps=chunk))
        if setup:
            setup(eng)
        eng.run(settle)
        st = torch.cuda.ExternalStream(eng.stream(), device=device)
        ev_c, sp_c, ms_c, hi_c = [], [], [], []
        fc_prev = eng.fire_count().astype(np.int64)
        done = 0
        while done < steps:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            i0 = eng.info().events_total
            e0.record(st)
            eng.run_async(chunk)
            e1.record(st)
            e1.synchronize()
            eng.sync()
            ms_c.append(e0.elapsed_time(e1))
            ev_c.append(eng.info().events_total - i0)
            fc = eng.fire_count().astype(np.int64)
            sp_c.append(int((fc - fc_prev).sum()))
            fc_prev = fc
            hi_c.append(((settle + done) // half) % 2 == 1)
            done += chunk
        stats = eng.predictor_stats() if deliv == B.DELIVERY_AUTO else None
        eng.close()
        return np.array(ev_c, np.float64), np.array(sp_c, np.float64), np.array(ms_c), np.array(hi_c), fc_prev, stats

    ev_p, sp_p, ms_p, hi_p, fc_p, _ = run_mode(B.DELIVERY_PUSH)
    ev_t, sp_t, ms_t, _, fc_t, _ = run_mode(B.DELIVERY_TILE)
    cost_push = PR.fit_costs(ev_p / chunk, ms_p * 1e6 / chunk)
    cost_tile = PR.fit_costs(ev_t / chunk, ms_t * 1e6 / chunk)

    def attach(eng):
        eng.enable_pop_stats(64)
        eng.set_predictor(params, tolerance=0.3, cost_push=cost_push, cost_tile=cost_tile)

    ev_a, _, ms_a, _, fc_a, st = run_mode(B.DELIVERY_AUTO, attach)

    def attach_exact(eng):
        eng.set_predictor(None, cost_push=cost_push, cost_tile=cost_tile)

    ev_x, _, ms_x, _, fc_x, st_x = run_mode(B.DELIVERY_AUTO, attach_exact)
    n_net = sp.n_pop * sp.pop_size
    rate = sp_p / chunk / n_net / DT
    eps = lambda ev, ms: float(ev.sum() / (ms.sum() / 1e3))
    frac = lambda ev, ms: roofline_frac(n_net * steps, float(ev.sum()), float(sp_p.sum()), float(ms.sum()) / 1e3)
    ideal = np.minimum(ms_p, ms_t).sum()  # the better fixed mode, chunk by chunk
    return {"workload": "predicted_2m: 200 x 10,000 LIF_brian, delays U{1..20}, 10 Hz square-wave i_offset; "
                        "%d cycles after %d settle cycles" % (steps, settle),
            "rate_hz_low_high": [float(rate[~hi_p].mean()) if (~hi_p).any() else None,
                                 float(rate[hi_p].mean()) if hi_p.any() else None],
            "events_per_s": {"push": eps(ev_p, ms_p), "tile": eps(ev_t, ms_t), "auto_predicted": eps(ev_a, ms_a),
                             "auto_exact": eps(ev_x, ms_x),
                             "best_fixed_per_chunk": float(ev_p.sum() / (ideal / 1e3))},
            "ms_per_cycle": {"push": float(ms_p.sum() / steps), "tile": float(ms_t.sum() / steps),
                             "auto_predicted": float(ms_a.sum() / steps), "auto_exact": float(ms_x.sum() / steps)},
            "hbm_roofline_frac": {"push": frac(ev_p, ms_p), "tile": frac(ev_t, ms_t), "auto_predicted": frac(ev_a, ms_a),
                                  "auto_exact": frac(ev_x, ms_x)},
            "cost_models_ns": {"push": cost_push, "tile": cost_tile, "form": "a + b * events per cycle"},
            "auto_exact_tile_cycles": int(st_x.tile_cycles),
            "spike_counts_identical": bool(np.array_equal(fc_p, fc_t) and np.array_equal(fc_p, fc_a)
                                           and np.array_equal(fc_p, fc_x)),
            "predictor": {"train_loss": loss, "train_seconds": t_train, "cycles": int(st.cycles),
                          "fallbacks": int(st.fallbacks), "fallback_rate": st.fallbacks / max(st.cycles, 1),
                          "tile_cycles": int(st.tile_cycles),
                          "rel_count_error": st.abs_err_sum / max(st.actual_sum, 1.0)}}


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def settle(eng, min_steps, max_steps, chunk=250, window=4, tol=0.03):
    """Runs the network out of its start-up transient before anything is timed: at
    least min_steps cycles, then chunks of `chunk` cycles until the mean events per
    cycle of the last `window` chunks is within `tol` of the `window` chunks before
    them (or max_steps). On the 1e6-neuron network the activity keeps rising for
    a few thousand cycles after the first spikes, so a fixed short settle would
    time a transient. Returns the cycles run and the events per cycle of each chunk."""
    per_chunk = []
    done = 0
    while True:
        e0 = eng.info().events_total
        eng.run(chunk)
        done += chunk
        per_chunk.append((eng.info().events_total - e0) / chunk)
        if done >= max_steps:
            break
        if done >= min_steps and len(per_chunk) >= 2 * window:
            a = np.mean(per_chunk[-window:])
            b = np.mean(per_chunk[-2 * window:-window])
            if abs(a - b) <= tol * max(a, 1.0):
                break
    return done, per_chunk


def dense_leg(steps, device, settle_min=1000):
    """The dense-firing configuration (50 x 20,000 LIF_brian, ~2 kHz, delays U{1..50}) as
    its own device-timed leg: events/s, realtime factor and the HBM roofline of its step."""
    import torch
    import bsim_b200 as B
    specs, desc = workload("dense_1m", 1)
    deliv = DEFAULT_DELIVERY.get("dense_1m", "push")
    eng = B.Engine.generated(specs, DT, opts=B.options(device=device, graph_steps=50, delivery={
        "push": B.DELIVERY_PUSH, "tile": B.DELIVERY_TILE}[deliv]))
    info = eng.info()
    N = info.n_neurons
    settled, _ = settle(eng, settle_min, 4 * settle_min, chunk=250, window=2)
    eng.run(5)
    st = torch.cuda.ExternalStream(eng.stream(), device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    i0 = eng.info().events_total
    fc0 = eng.fire_count().astype(np.int64)
    e0.record(st)
    eng.run_async(steps)
    e1.record(st)
    e1.synchronize()
    eng.sync()
    ms = e0.elapsed_time(e1)
    ev = eng.info().events_total - i0
    spk = int((eng.fire_count().astype(np.int64) - fc0).sum())
    eng.close()
    peak, _ = measured_hbm_peak()
    alg = BYTES_PER_NEURON_STEP * N + BYTES_PER_EVENT * ev / steps + BYTES_PER_SPIKE * spk / steps
    ach = alg / (ms / steps / 1e3) / 1e9
    return {"workload": "dense_1m: " + desc, "neurons": N, "synapses": int(info.n_synapses), "delivery": deliv,
            "settle_steps": settled, "steps": steps, "ms_per_step": ms / steps, "events_per_s": ev / (ms / 1e3),
            "events_per_step": ev / steps, "mean_rate_hz": spk / N / (steps * DT),
            "realtime_factor": steps * DT / (ms / 1e3),
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "alg_bytes_per_launch": alg}}


def reference_program_leg(depth=120, n=1000, preset=("0.7", "0.5", "0.6", "0.3", "6")):
    """The reference's own benchmark program, test/gpu/standard_test.cpp, compiled unchanged
    against include/BSim.h (oracle/_ref/progs, built where the reference's sources are
    present), run on the case its source comments time on a P100: depth 120, 1,000
    neurons per population, the 2 % preset, 1,000 cycles. Its GSim.info loop time (the
    same gettimeofday window as the reference's) is set beside the published 0.432303 s
    (test/gpu/standard_test.cpp:22,29-30,43; other hardware, depth unspecified there
    within 120-300)."""
    prog = os.path.join(ROOT, "oracle", "_ref", "progs", "standard_test")
    if not os.path.exists(prog):
        return {"unavailable": "the reference's programs were not built (no reference sources at build time)"}
    out = {"program": "standard_test %d %d %s" % (depth, n, " ".join(preset)), "cycles": 1000,
           "p100_published_loop_seconds": 0.432303}
    for deliv in ("push", "tile"):
        with tempfile.TemporaryDirectory() as d:
            env = dict(os.environ, BSIM_DELIVERY=deliv)
            t0 = time.perf_counter()
            r = subprocess.run([prog, str(depth), str(n)] + list(preset), cwd=d, env=env, capture_output=True,
                               text=True, timeout=600)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                out[deliv] = {"error": r.stderr[-300:]}
                continue
            info = open(os.path.join(d, "GSim.info")).read()
            loop = None
            for line in info.splitlines():
                if line.startswith("Simulation fin"):
                    h, m, sec = line.rsplit(" in ", 1)[1].strip().rstrip("s").split(":")
                    loop = 3600 * int(h) + 60 * int(m) + float(sec)
            counts = np.loadtxt(os.path.join(d, "GFire.count"), dtype=np.int64)
            out[deliv] = {"loop_seconds": loop, "program_wall_seconds": wall,
                          "speedup_vs_p100": 0.432303 / loop if loop else None,
                          "spikes": int(counts.sum()), "neurons": int(counts.shape[0]),
                          "info": " ".join(info.split())[:200]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--config", default="plain_1m")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--delivery", default=None, choices=["push", "pull", "tile", "auto"],
                    help="default: the fastest measured mode of the workload (DEFAULT_DELIVERY)")
    ap.add_argument("--settle", type=int, default=3000,
                    help="untimed cycles run at set-up at least, so the network leaves its start-up transient")
    ap.add_argument("--settle-max", type=int, default=10000,
                    help="settling stops here even if the activity is still drifting")
    ap.add_argument("--dense-steps", type=int, default=200,
                    help="timed cycles of the dense-firing leg (50 x 20,000, ~2 kHz, delays 1-50; 0 skips it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-program", action="store_true",
                    help="skip the reference's standard_test program (depth 120, 1,000 neurons, 2 %% preset)")
    ap.add_argument("--batched-nets", type=int, default=256,
                    help="networks in the batched+predicted vs plain comparison (0 skips it)")
    ap.add_argument("--batched-steps", type=int, default=500)
    ap.add_argument("--predicted-steps", type=int, default=2000,
                    help="cycles of the predictor-scheduled comparison (0 skips it)")
    args = ap.parse_args()
    if args.delivery is None:
        args.delivery = DEFAULT_DELIVERY.get(args.config, "push")
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import bsim_b200 as B

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        # every rank does the same work between collectives (seconds): a rank that dies or
        # never arrives ends the others' next collective with an error after this bound
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))

    specs, desc = workload(args.config, 1 + rank)
    deliv = {"push": B.DELIVERY_PUSH, "pull": B.DELIVERY_PULL, "tile": B.DELIVERY_TILE,
             "auto": B.DELIVERY_AUTO}[args.delivery]
    t_build = time.perf_counter()
    # cycles replayed from CUDA graphs of up to 100 launches; a timed run of K <= 100 cycles is
    # one graph (captured while the network settles), not K separate launches
    eng = B.Engine.generated(specs, DT, opts=B.options(device=local, delivery=deliv,
                                                       graph_steps=max(1, min(100, args.steps))))
    t_build = time.perf_counter() - t_build
    info = eng.info()
    N, S = info.n_neurons, info.n_synapses

    settled = settle(eng, args.settle, args.settle_max)
    eng.run(args.warmup)
    stream = torch.cuda.ExternalStream(eng.stream(), device=local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    i0 = eng.info()
    fc0 = eng.fire_count().astype(np.int64)
    with ClockSampler(local) as clk:
        e0.record(stream)
        eng.run_async(args.steps)
        e1.record(stream)
        clk.poll_until(e1)  # clocks sampled while the timed steps run
    eng.sync()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    i1 = eng.info()
    events = int(i1.events_total - i0.events_total)
    spikes = int((eng.fire_count().astype(np.int64) - fc0).sum())
    (ms_max,), (events_all, spikes_all, n_all) = reduce_over_ranks(dist, [ms], [events, spikes, N], "cuda")
    value = events_all / (ms_max / 1e3)
    rtf = args.steps * DT / (ms_max / 1e3)
    ms_step = ms_max / args.steps

    # end to end through the C ABI with host buffers: upload the neuron state,
    # run the steps recording every spike, read the raster and the counts back
    st = eng.state()
    e2e_steps = args.steps
    cap = int(max(4 * spikes, 1024))
    # page-locked host buffers, allocated once outside the timed region as a
    # streaming user would: the state to upload and the raster to read back into
    def pinned(a):
        try:
            return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        except RuntimeError:  # page-locked memory refused: the pageable copy still works
            return np.ascontiguousarray(a)
    v, ie, ii, rf = pinned(st["v"]), pinned(st["i_E"]), pinned(st["i_I"]), pinned(st["refrac"])
    n_ras = int(1.25 * spikes * e2e_steps / args.steps) + 1024
    try:
        ras_buf = torch.empty(n_ras, dtype=torch.int32, pin_memory=True).numpy()
        cnt_buf = torch.empty(N, dtype=torch.int32, pin_memory=True).numpy()
    except RuntimeError:
        ras_buf = np.empty(n_ras, np.int32)
        cnt_buf = np.empty(N, np.int32)
    eng.record(e2e_steps, cap)  # allocates the recording buffers (drops the captured graph)
    eng.run(100)                # re-captures the graph with recording enabled (not timed)
    # one untimed pass of the whole path first, so that the timed one does not pay for
    # loading the kernels it launches for the first time (the state packing, the raster's
    # flush and sort)
    eng.record(e2e_steps, cap)
    eng.write_state(v, ie, ii, rf)
    eng.run(e2e_steps)
    eng.raster(out=ras_buf)
    eng.fire_count(out=cnt_buf)
    eng.record(e2e_steps, cap)  # re-arms the recording only
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ia = eng.info()
    t0 = time.perf_counter()
    eng.write_state(v, ie, ii, rf)
    t1 = time.perf_counter()
    eng.run(e2e_steps)
    t2 = time.perf_counter()
    raster = eng.raster(out=ras_buf)
    t3 = time.perf_counter()
    counts = eng.fire_count(out=cnt_buf)
    t4 = time.perf_counter()
    t_e2e = t4 - t0
    parts_ms = {"write_state": 1e3 * (t1 - t0), "run": 1e3 * (t2 - t1), "raster": 1e3 * (t3 - t2),
                "fire_count": 1e3 * (t4 - t3)}
    ib = eng.info()
    ev_e2e = float(ib.events_total - ia.events_total)
    spk_e2e = sum(len(r) for r in raster)
    (t_e2e_max,), (ev_all_e2e,) = reduce_over_ranks(dist, [t_e2e], [ev_e2e], "cuda")
    e2e = {"value": ev_all_e2e / t_e2e_max, "unit": "events/s",
           "h2d_bytes_per_step": 16.0 * N / e2e_steps,
           "d2h_bytes_per_step": (4.0 * spk_e2e + 8.0 * (e2e_steps + 1) + 4.0 * len(counts)) / e2e_steps,
           "realtime_factor": e2e_steps * DT / t_e2e_max, "steps": e2e_steps,
           "parts_ms": parts_ms,
           "path": "bsim_write_state (H2D from page-locked buffers) + bsim_run with spike recording + "
                   "bsim_read_raster (into a page-locked buffer) + bsim_read_fire_count (D2H into a "
                   "page-locked buffer), wall clock, each call synchronous"}

    peak, peak_kind = measured_hbm_peak()
    alg_bytes = (BYTES_PER_NEURON_STEP * N + BYTES_PER_EVENT * events / args.steps +
                 BYTES_PER_SPIKE * spikes / args.steps)
    achieved = alg_bytes / (ms / args.steps / 1e3) / 1e9
    traffic = profiled_traffic(args.config, args.delivery, alg_bytes)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
            if peak_kind == "measured" else "fallback 6.65 TB/s",
            "kernel": "step_kernel<EXACT> (fused LIF update + %s delivery), one launch per step" % args.delivery,
            "alg_bytes_per_launch": alg_bytes}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            eps, ci = cpu_baseline(specs[0], 300)
            cpu = {"value": eps, "unit": "events/s", "cores": 1, "kind": ci["kind"], "sample": ci["sample"],
                   "realtime_factor_of_sample": ci["rtf"]}
        except Exception as ex:
            cpu = {"value": None, "unit": "events/s", "cores": 1, "kind": "unavailable", "sample": str(ex)}

    eng.close()  # frees the timed network before the comparisons build theirs
    cmp = None
    if rank == 0 and world == 1 and args.batched_nets > 0:
        try:
            cmp = batched_vs_plain(args.batched_nets, args.batched_steps, local)
        except Exception as ex:
            cmp = {"error": str(ex)}
    dense = None
    if rank == 0 and world == 1 and args.dense_steps > 0:
        try:
            dense = dense_leg(args.dense_steps, local)
        except Exception as ex:
            dense = {"error": str(ex)}
    refprog = None
    if rank == 0 and world == 1 and not args.no_reference_program:
        try:
            refprog = reference_program_leg()
        except Exception as ex:
            refprog = {"error": str(ex)}
    pred = None
    if rank == 0 and world == 1 and args.predicted_steps > 0:
        try:
            pred = predicted_vs_plain(args.predicted_steps, local)
        except Exception as ex:
            pred = {"error": str(ex)}

    if rank == 0:
        line = {"metric": "synaptic events/s", "value": value, "unit": "events/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: seeded generator, networks built on the device",
                "config": {"workload": args.config + ": " + desc, "neurons_per_gpu": N, "synapses_per_gpu": S,
                           "delivery": args.delivery, "accumulate": "exact int64",
                           "parallelism": "replicas x%d (independent networks, no collective)" % world,
                           "l2": "inputs larger than L2 (%.1f GB of synapse rows per GPU)" % (S * 8 / 1e9),
                           "build_seconds": t_build, "settle_steps": settled[0],
                           "settle_events_per_cycle_last_chunks": [float(x) for x in settled[1][-8:]]},
                "realtime_factor": rtf, "spikes_per_step": spikes_all / args.steps / world,
                "events_per_step": events_all / args.steps / world,
                "mean_rate_hz": spikes_all / n_all / (args.steps * DT),
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
                "gpu_launches": args.steps, "dense_c2": dense, "reference_program_standard_test": refprog, "batched_vs_plain": cmp,
                "predictor_scheduled_vs_plain": pred}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
