"""Batched scene pipeline: build + query many uneven scenes as one CUDA graph.

A BatchPipeline owns one Batch per primitive kind (triangle scenes, point scenes), one
BatchPlan per query operation, the device inputs and outputs, and the launch shapes the
autotuner chose.  `capture()` records the whole step -- both builds and every query phase,
the triangle and point branches on two streams -- into one CUDA graph; `replay()` runs it.
`run_loop()` runs the same work as a per-scene loop over the single-tree calls (the
comparison schedule); `results()` reads every output back for comparison.

Every phase of the graph is one launch over all scenes of its kind (qk_batch_* in
libquarry_b200.so); nothing in the step synchronizes with the host.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import autotune, capi

OPS = {"rays": capi.QK_OP_RAY, "closest": capi.QK_OP_CLOSEST, "knn": capi.QK_OP_KNN,
       "radius": capi.QK_OP_RADIUS}


@dataclass
class Phase:
    kind: str          # "tri" | "point"
    name: str          # "rays" | "closest" | "knn" | "radius"
    counts: np.ndarray
    inputs: object     # device tensor
    out: object
    offsets: object
    capacity: int
    params: dict       # autotuned point (flags + launch shape)
    plans: dict        # flags -> BatchPlan


class BatchPipeline:
    def __init__(self, terrains: list, clouds: list, k: int = 16):
        import torch

        self.torch = torch
        self.k = k
        self.scenes = {"tri": terrains, "point": clouds}
        self.batches = {}
        self.phases: list[Phase] = []
        self.radii = {kind: np.array([s.r for s in sc], np.float32)
                      for kind, sc in self.scenes.items() if sc}
        self.wide = {kind: True for kind in self.scenes}
        self._make_batches()
        for kind, sc in self.scenes.items():
            if not sc:
                continue
            names = (["rays"] if kind == "tri" else []) + ["closest", "knn", "radius"]
            for name in names:
                parts = [getattr(s, name) for s in sc]
                counts = np.array([p.shape[0] for p in parts], np.int32)
                inputs = capi.to_device(np.concatenate(parts, axis=0), np.float32)
                n = int(counts.sum())
                dev = "cuda"
                offsets = None
                if name == "rays":
                    out = torch.empty(n, dtype=torch.int64, device=dev)
                elif name == "closest":
                    out = torch.empty((n, 2), dtype=torch.int32, device=dev)
                elif name == "knn":
                    out = torch.empty((n, k, 2), dtype=torch.int32, device=dev)
                else:
                    out = torch.empty(1, dtype=torch.int64, device=dev)
                    offsets = torch.empty(n + len(sc) + 1, dtype=torch.int32, device=dev)
                self.phases.append(Phase(kind, name, counts, inputs, out, offsets, 0,
                                         dict(autotune.BATCH_START), {}))
        self.graph = None
        self.streams = None
        self.builder = "lbvh"   # or "sah<bins>": per-scene SAH builds, outside the graph

    # ---- objects ----
    def build_trees(self, kind: str) -> None:
        if self.builder == "lbvh":
            self.batches[kind].build()
        else:
            self.batches[kind].build_sah(int(self.builder[3:]))

    def _make_batches(self):
        for kind, sc in self.scenes.items():
            if sc:
                self.batches[kind] = capi.Batch(kind, [s.items for s in sc], wide=self.wide[kind])
                self.batches[kind].build()
                self.batches[kind].sync()

    def plan(self, ph: Phase, flags: int) -> capi.BatchPlan:
        if flags not in ph.plans:
            params = self.radii[ph.kind] if ph.name == "radius" else None
            ph.plans[flags] = self.batches[ph.kind].plan(OPS[ph.name], ph.counts, params, flags)
        return ph.plans[flags]

    def size_radius_outputs(self) -> None:
        """Counts every radius phase once (untimed) and sizes its key buffer to fit."""
        torch = self.torch
        for ph in self.phases:
            if ph.name != "radius":
                continue
            p = self.plan(ph, ph.params["flags"])
            p.query(ph.inputs, ph.out, offsets=ph.offsets, capacity=0)
            total, _ = p.status(raise_on_overrun=False)
            ph.capacity = int(total)
            ph.out = torch.empty(max(total, 1), dtype=torch.int64, device="cuda")

    def run_phase(self, ph: Phase, params: dict | None = None,
                  schedule: int = capi.QK_SCHEDULE_BATCHED) -> None:
        params = params or ph.params
        p = self.plan(ph, params["flags"])
        tune = autotune.batch_launch(params) if schedule == capi.QK_SCHEDULE_BATCHED else None
        p.query(ph.inputs, ph.out, offsets=ph.offsets, capacity=ph.capacity, k=self.k,
                tune=tune, schedule=schedule)

    def fingerprint(self, ph: Phase) -> tuple:
        """Device checksum of a phase's outputs (autotuner result check)."""
        torch = self.torch
        parts = [ph.out.view(torch.int64).flatten()]
        if ph.offsets is not None:
            parts.append(ph.offsets[: int(ph.counts.sum()) + 1].to(torch.int64))
        out = []
        for v in parts:
            w = torch.arange(1, 2 * v.numel() + 1, 2, dtype=torch.int64, device=v.device)
            out += [int(v.sum()), int((v * w).sum()), int((v ^ (v >> 17)).sum())]
        return tuple(out)

    # ---- tuning ----
    def signature(self, ph: Phase) -> str:
        n = int(sum(s.items.shape[0] for s in self.scenes[ph.kind]))
        return (f"batch:{ph.kind}:{ph.name}:scenes={len(ph.counts)}:prims={n}:"
                f"queries={int(ph.counts.sum())}:k={self.k}:space=3")

    def tune(self, tuner: autotune.Autotuner, force: bool = False, repeats: int = 3) -> dict:
        report = {}
        for ph in self.phases:
            def run(params, ph=ph):
                self.run_phase(ph, params)

            res = tuner.search(self.signature(ph), autotune.BATCH_SPACE, run,
                               fingerprint=lambda params, ph=ph: self.fingerprint(ph),
                               start=autotune.BATCH_START, valid=autotune.batch_valid(ph.name),
                               repeats=repeats, force=force)
            ph.params = dict(res.params)
            report[f"{ph.kind}_{ph.name}"] = {"params": res.params, "ms": round(res.ms, 4),
                                              "cached": res.cached, "source": res.source,
                                              "tuning_s": round(res.tuning_s, 2),
                                              "points": len(res.trials)}
        tuner.save()
        # a batch whose phases all chose the binary layout is rebuilt without 4-wide nodes
        for kind in list(self.batches):
            uses_wide = any(ph.params["flags"] & capi.QK_WIDE for ph in self.phases
                            if ph.kind == kind)
            if not uses_wide and self.wide[kind]:
                self.wide[kind] = False
                self.batches[kind] = capi.Batch(kind, [s.items for s in self.scenes[kind]],
                                                wide=False)
                self.batches[kind].build()
                self.batches[kind].sync()
                for ph in self.phases:
                    if ph.kind == kind:
                        ph.plans = {}
        return report

    # ---- schedules ----
    def step(self, streams=None) -> None:
        """One batched step on the current stream (or tri / point on two streams)."""
        torch = self.torch
        kinds = [k for k in ("tri", "point") if k in self.batches]
        main = torch.cuda.current_stream()
        in_graph = self.builder == "lbvh"
        if streams is None:
            for kind in kinds:
                self.build_trees(kind)
                for ph in self.phases:
                    if ph.kind == kind:
                        self.run_phase(ph)
            return
        for s in streams:
            s.wait_stream(main)
        for kind, s in zip(kinds, streams):
            with torch.cuda.stream(s):
                if in_graph:
                    self.batches[kind].build()
                for ph in self.phases:
                    if ph.kind == kind:
                        self.run_phase(ph)
        for s in streams:
            main.wait_stream(s)

    def capture(self) -> None:
        """Records one batched step (both kinds on two forked streams) as a CUDA graph."""
        torch = self.torch
        for ph in self.phases:  # plans exist before capture (their creation synchronizes)
            self.plan(ph, ph.params["flags"])
        cap = torch.cuda.Stream()
        self.streams = (torch.cuda.Stream(), torch.cuda.Stream())
        cap.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(cap):
            self.step(self.streams)  # warm-up outside the graph
        torch.cuda.current_stream().wait_stream(cap)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph(keep_graph=True)
        with torch.cuda.graph(self.graph, stream=cap):
            self.step(self.streams)
        self.kernel_nodes = self._count_kernel_nodes()
        self.graph.instantiate()
        torch.cuda.synchronize()

    def replay(self) -> None:
        """One step: the graph (builds included with the batched LBVH); per-scene SAH builds,
        which synchronize, run before it."""
        if self.builder != "lbvh":
            for kind in self.batches:
                self.build_trees(kind)
        self.graph.replay()

    def tune_builder(self, tuner: autotune.Autotuner, force: bool = False,
                     repeats: int = 2) -> dict:
        """Chooses the builder (batched LBVH, or per-scene SAH with 8 / 16 / 32 bins) by the
        time of a whole step: every build plus every query phase with its tuned shape."""
        sig = "batch-step:" + "|".join(self.signature(ph) for ph in self.phases)

        def run(params):
            self.builder = params["builder"]
            self.step()

        def fp(params):
            return tuple(self.fingerprint(ph) for ph in self.phases)

        res = tuner.search(sig, {"builder": ["lbvh", "sah8", "sah16", "sah32"]}, run,
                           fingerprint=fp, start={"builder": "lbvh"}, repeats=repeats,
                           force=force, tolerance=0.0)
        self.builder = res.params["builder"]
        for kind in self.batches:
            self.build_trees(kind)
            self.batches[kind].sync()
        tuner.save()
        return {"params": res.params, "ms": round(res.ms, 3), "cached": res.cached,
                "source": res.source, "points": [(t["params"]["builder"], t["ms"])
                                                 for t in res.trials]}

    def graph_kernel_nodes(self) -> int | None:
        """Kernel nodes in the captured graph (None when the runtime bindings are missing)."""
        return getattr(self, "kernel_nodes", None)

    def _count_kernel_nodes(self) -> int | None:
        try:
            from cuda.bindings import runtime as rt

            g = self.graph.raw_cuda_graph()
            g = rt.cudaGraph_t(init_value=int(g)) if not isinstance(g, rt.cudaGraph_t) else g
            err, _, n = rt.cudaGraphGetNodes(g, 0)
            if err != rt.cudaError_t.cudaSuccess:
                return None
            err, nodes, n = rt.cudaGraphGetNodes(g, n)
            if err != rt.cudaError_t.cudaSuccess:
                return None
            count = 0
            for node in nodes[:n]:
                err, t = rt.cudaGraphNodeGetType(node)
                if err == rt.cudaError_t.cudaSuccess and \
                        t == rt.cudaGraphNodeType.cudaGraphNodeTypeKernel:
                    count += 1
            return count
        except Exception:
            return None

    def run_loop(self) -> None:
        """The same step as a per-scene loop over the single-tree calls."""
        for kind in ("tri", "point"):
            if kind not in self.batches:
                continue
            if self.builder == "lbvh":
                self.batches[kind].build(capi.QK_SCHEDULE_LOOP)
            else:
                self.build_trees(kind)
            for ph in self.phases:
                if ph.kind == kind:
                    self.run_phase(ph, schedule=capi.QK_SCHEDULE_LOOP)

    def sync(self) -> None:
        for b in self.batches.values():
            b.sync()
        for ph in self.phases:
            self.plan(ph, ph.params["flags"]).status()

    # ---- read-back ----
    def results(self, loop_layout: bool = False) -> dict:
        """Per phase: per-scene host results.  Radius results are (offsets, keys) per scene;
        loop_layout reads the radius CSR in the loop schedule's per-scene layout."""
        out = {}
        for ph in self.phases:
            q_off = np.concatenate([[0], np.cumsum(ph.counts)]).astype(np.int64)
            if ph.name == "radius":
                off = ph.offsets.cpu().numpy().astype(np.int64)
                keys = ph.out.cpu().numpy().view(np.uint64)
                per, base = [], 0
                for i in range(len(ph.counts)):
                    q0, q1 = q_off[i], q_off[i + 1]
                    if loop_layout:
                        o = off[q0 + i:q1 + i + 1]
                        k = keys[base:base + int(o[-1])]
                        base += int(o[-1])
                    else:
                        o = off[q0:q1 + 1] - off[q0]
                        k = keys[off[q0]:off[q1]]
                    per.append((o.copy(), k.copy()))
            else:
                a = ph.out.cpu().numpy()
                a = a.view(np.uint64) if ph.name == "rays" else a.view(np.uint32)
                per = [a[q_off[i]:q_off[i + 1]] for i in range(len(ph.counts))]
            out[f"{ph.kind}_{ph.name}"] = per
        return out

    def query_count(self) -> int:
        return int(sum(int(ph.counts.sum()) for ph in self.phases))
