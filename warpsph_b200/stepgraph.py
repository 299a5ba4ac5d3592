"""Whole integrator steps recorded once as a CUDA graph and replayed.

One RK2 step of the compressible schemes (schemes/crkSPH.py:19-366, compSPH) issues
about fifty kernel launches from Python, and the host-side keep-or-rebuild decision of
the neighbour list reads the device in every stage.  On 10^5..10^6 particles the host
work is as long as the GPU work, so the GPU waits on the interpreter.

``StepGraph`` removes both:
  * the step runs with device-decided neighbour lists (``ops.device_decided_lists``): the
    Verlet rows live in fixed buffers and the GPU itself keeps or rebuilds them, so no
    step reads the device;
  * one whole step (the CFL time step, every stage, the compatible-energy finalize) is
    recorded into a CUDA graph whose last nodes copy the new state into the graph's
    input buffers, and each further step is one graph launch.

Usage::

    sg = StepGraph(system, integrator, step_fn, config, compParams, dt=config.dt)
    sg.replay(100)                 # 100 steps, no host work beyond the launches
    sg.check()                     # one host read: list overflow / bad supports
    state = sg.system.state        # tensors the next replay overwrites (clone to keep)

The neighbour list has a fixed capacity, 1.3 times the entries of one build at the start
(``ops.DEVICE_LIST_HEADROOM``); a workload whose neighbour counts grow past it makes
``check()`` raise, and is recorded again with a larger headroom from a saved state.

Each step's time step is ``next_dt(system, dt_prev)`` (a device scalar); the default is
the CFL step of the compressible schemes (modules/timestep/compressible.py:12-66) when
``config.adaptiveDt`` is set, else the fixed dt.  The step function must not read the
device (schemes whose solvers test convergence on the host, such as DFSPH, cannot be
recorded; torch raises during the recording).  The state a replay leaves is the one an
eager run with device-decided lists gives, up to the summation order of the pair sums.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Optional

import torch

from . import _capi, ops
from .configurations import make_params


def _cfl_next_dt(config, compParams):
    params = make_params(config, compParams)

    def next_dt(system, dt_prev):
        S = system.state
        return ops.cfl_dt(params, S.supports, S.internalEnergies, dt_prev=dt_prev)
    return next_dt


def _per_particle(state, n: int):
    """(name, tensor) of the state's per-particle tensors (first dimension n)."""
    out = []
    for f in dataclasses.fields(state):
        v = getattr(state, f.name)
        if isinstance(v, torch.Tensor) and v.dim() >= 1 and v.shape[0] == n:
            out.append((f.name, v))
    return out


class StepGraph:
    """A recorded integrator step over one particle system (see the module docstring).

    system: the system to advance; its state is copied into the graph's input buffers
        after ``warmup`` eager steps (so the first replay continues from the state those
        steps reach, ``warmup`` steps after ``system``);
    integrator, step_fn, config, compParams: as for ``integrator.function``;
    dt: the previous (or fixed) time step, a float or a device scalar;
    next_dt: optional ``(system, dt_prev) -> device scalar``."""

    def __init__(self, system, integrator, step_fn, config, compParams, dt, warmup: int = 3,
                 next_dt: Optional[Callable] = None):
        dev = system.state.positions.device
        self.device = dev
        self.integrator, self.step_fn, self.config, self.compParams = integrator, step_fn, config, compParams
        if next_dt is None:
            if getattr(config, "adaptiveDt", False):
                next_dt = _cfl_next_dt(config, compParams)
            else:
                next_dt = lambda system, dt_prev: dt_prev   # noqa: E731
        self.next_dt = next_dt
        n = int(system.state.positions.shape[0])
        self.n = n
        dt_t = ops.dt_tensor(dt, dev).clone()
        if ops.TIMER is not None:
            raise RuntimeError("StepGraph: stop the kernel timer (ops.TIMER) before recording")

        launches0 = _capi.lib().sph_launch_count()
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with ops.device_decided_lists(), torch.cuda.stream(side):
            for _ in range(max(int(warmup), 1)):
                system, dt_t = self._advance(system, dt_t)
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self.warmup_launches = _capi.lib().sph_launch_count() - launches0
        self.lists = [nb for key, nb in ops._device_lists.items() if key[0] == dev.index and key[1] == n]
        for nb in self.lists:
            nb.check()

        # the graph's input buffers: copies of every per-particle tensor of the state
        self.inputs = system.initializeNewState()
        for name, v in _per_particle(system.state, n):
            setattr(self.inputs.state, name, v.clone())
        t_dev = getattr(system, "t_device", None)
        if isinstance(t_dev, torch.Tensor):
            self.inputs.t_device = t_dev.clone()
        self.dt = dt_t.clone()

        self.graph = torch.cuda.CUDAGraph()
        lib = _capi.lib()
        launches0, cond0 = lib.sph_launch_count(), lib.sph_launch_count_conditional()
        gen0 = [nb.generation for nb in self.lists]
        # thread-local capture: other threads of the process (a process group's watchdog, for
        # one) may keep making CUDA calls while this thread records
        with ops.device_decided_lists(), torch.cuda.graph(self.graph, capture_error_mode="thread_local"):
            out, dt_new = self._advance(self.inputs, self.dt)
            static = dict(_per_particle(self.inputs.state, n))
            dsts, srcs = [], []
            for name, v in _per_particle(out.state, n):
                dst = static.get(name)
                if dst is None:
                    raise RuntimeError(f"StepGraph: the step produces state field {name!r} that the warm-up state lacks")
                if dst is not v:
                    dsts.append(dst)
                    srcs.append(v)
            if dsts:
                torch._foreach_copy_(dsts, srcs)     # the copies in one or a few multi-tensor launches
            self.dt.copy_(dt_new)
            if isinstance(getattr(out, "t_device", None), torch.Tensor) and isinstance(getattr(self.inputs, "t_device", None), torch.Tensor):
                self.inputs.t_device.copy_(out.t_device)
        # this library's kernels in one recorded step: those every replay runs, and those of
        # one neighbour-list rebuild (the bodies of the rebuild conditionals)
        cond = lib.sph_launch_count_conditional() - cond0
        updates = sum(nb.generation - g for nb, g in zip(self.lists, gen0))
        self.launches_per_step = lib.sph_launch_count() - launches0 - cond
        self.launches_per_rebuild = cond // updates if updates and cond else 0
        self.out = out
        self.steps = 0

    def _advance(self, system, dt_prev):
        dt = self.next_dt(system, dt_prev)
        res = self.integrator.function(state=system, f=self.step_fn, dt=dt, config=self.config, compParams=self.compParams)
        return res.state, dt

    @property
    def system(self):
        """The system after the latest replay (graph-owned tensors; clone what you keep)."""
        return self.out

    def replay(self, steps: int = 1) -> None:
        """Launches `steps` recorded steps on the current stream."""
        for _ in range(int(steps)):
            self.graph.replay()
        self.steps += int(steps)

    def load_state(self, fields: dict) -> None:
        """Copies tensors (device or pinned host, by state field name) into the graph's input
        buffers, on the current stream; the next replay starts from them."""
        names = list(fields)
        dsts = [getattr(self.inputs.state, name) for name in names]
        srcs = [fields[name] for name in names]
        if all(t.is_cuda for t in srcs):
            torch._foreach_copy_(dsts, srcs, non_blocking=True)   # one multi-tensor launch
        else:
            for d, v in zip(dsts, srcs):
                d.copy_(v, non_blocking=True)

    def rebuilds(self) -> int:
        """Neighbour-list rebuilds so far (counted on the device; one host read per list)."""
        return sum(int(nb.rebuilds.item()) for nb in self.lists)

    def check(self) -> None:
        """Raises if a neighbour-list rebuild since the start overflowed the list or met a
        non-finite support (one host read per list)."""
        for nb in self.lists:
            nb.check()

    def release(self) -> None:
        self.graph.reset()
        self.out = None
