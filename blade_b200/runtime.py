"""Pipeline, Runner and the Python entry points bl.module / bl.runner.

Mirrors:
* ``Blade::Pipeline`` (include/blade/pipeline.hh:15-89, src/pipeline.cc:7-141):
  two non-blocking streams, module registration with CHRONOUS compute-ratio
  stepping, ``compute(index)``, ``synchronize``, ``is_synchronized``, ``will_output``;
* ``Blade::Runner`` (include/blade/runner.hh:14-52, src/runner.cc:7-68): the
  two-slot asynchronous queue (``enqueue``/``dequeue``/``copy``);
* ``bl.module`` (python/blade/_modules/__init__.py:5-148) and ``bl.runner``
  (python/blade/_runner/__init__.py:6-86).

Differences by design: every module output is allocated per slot, so the two
in-flight slots never share an intermediate buffer; and with ``graph=True`` the
steady-state ``compute(index)`` of each slot is captured once into a CUDA graph
and replayed (one graph launch per block instead of one launch per module).
"""

from __future__ import annotations

import contextlib
import threading
from collections import deque
from types import SimpleNamespace

import torch

from . import constants as K
from .constants import Constant, Taint, result
from .memory import Duet, Vector, as_vector, copy as _copy
from .modules import REGISTRY, Module

_tls = threading.local()


def _fetch_pipeline():
    """The pipeline under construction on this thread (the reference's frame-walking
    ``_Fetch``, python/blade/_internal/__init__.py:10-41)."""
    stack = getattr(_tls, "stack", None)
    return stack[-1] if stack else None


@contextlib.contextmanager
def _building(pipeline):
    stack = getattr(_tls, "stack", None)
    if stack is None:
        stack = _tls.stack = []
    stack.append(pipeline)
    try:
        yield
    finally:
        stack.pop()


class _HostStream:
    """Stand-in stream when no CUDA device is present (host-side logic only)."""

    cuda_stream = None

    def synchronize(self):
        pass

    def query(self):
        return True


class Pipeline:
    """Ordered module chain over two CUDA streams."""

    def __init__(self, graph: bool = False):
        if torch.cuda.is_available():
            self._streams = [torch.cuda.Stream(), torch.cuda.Stream()]
        else:
            self._streams = [_HostStream(), _HostStream()]
        self._modules: list[Module] = []
        self._commited = False
        self._step = 0
        self._steps_per_cycle = 1
        self._lifetime_cycles = 0
        self._ratios: list[int] = []
        self._graph_enabled = graph
        self._graphs: dict[int, torch.cuda.CUDAGraph] = {}
        self._warm: dict[int, int] = {}

    # -- reference surface -----------------------------------------------------
    def compute_complete(self) -> bool:
        return self._step + 1 == self._steps_per_cycle

    def compute_current_step_count(self) -> int:
        return self._step

    def compute_steps_per_cycle(self) -> int:
        return self._steps_per_cycle

    def compute_lifetime_cycles(self) -> int:
        return self._lifetime_cycles

    def commited(self) -> bool:
        return self._commited

    def will_output(self) -> bool:
        return self._steps_per_cycle == self._step + 1

    def stream(self, index: int = 0) -> torch.cuda.Stream:
        return self._streams[index]

    def number_of_streams(self) -> int:
        return len(self._streams)

    def add_module(self, module: Module) -> None:
        """src/pipeline.cc:22-39."""
        if self._commited:
            raise RuntimeError("Can't connect new module after Pipeline is commited.")
        if (module.get_taint() & Taint.CHRONOUS) == Taint.CHRONOUS:
            r = module.get_compute_ratio()
            if r > 1:
                self._steps_per_cycle *= r
                self._ratios.append(r)
        self._modules.append(module)

    def _commit(self):
        self._ratios.append(1)
        self._commited = True

    def _run_modules(self, index: int) -> result:
        """src/pipeline.cc:89-141: each module's process() with CHRONOUS stepping."""
        stream = self._streams[index]
        local_offset, ratio_index = 1, 0
        for m in self._modules:
            m._set_slot(index)
        for m in self._modules:
            local_step = self._step // local_offset % self._ratios[ratio_index]
            res = m.process(local_step, stream)
            if res == result.pipeline_exhausted:
                return res
            if res != result.success:
                return res
            if m.get_compute_ratio() > 1:
                if local_step == self._ratios[ratio_index] - 1:
                    local_offset += local_step
                    ratio_index += 1
                else:
                    break
        return result.success

    def compute(self, index: int) -> result:
        if not self._commited:
            self._commit()
        use_graph = self._graph_enabled and self._steps_per_cycle == 1
        if use_graph and index in self._graphs:
            for m in self._modules:
                m._set_slot(index)
            with torch.cuda.stream(self._streams[index]):
                self._graphs[index].replay()
            res = result.success
        elif use_graph and self._warm.get(index, 0) >= 1:
            # Capture the steady state of this slot once (after one eager run, so
            # every one-time setup such as shared-memory opt-ins has happened).
            g = torch.cuda.CUDAGraph()
            self._streams[index].synchronize()
            with torch.cuda.graph(g, stream=self._streams[index], capture_error_mode="thread_local"):
                res = self._run_modules(index)
            self._graphs[index] = g
            with torch.cuda.stream(self._streams[index]):
                g.replay()
        else:
            res = self._run_modules(index)
            self._warm[index] = self._warm.get(index, 0) + 1
        if res != result.success:
            return res
        self._step += 1
        if self._step == self._steps_per_cycle:
            self._step = 0
            self._lifetime_cycles += 1
        return result.success

    def synchronize(self, index: int) -> result:
        self._streams[index].synchronize()
        return result.success

    def is_synchronized(self, index: int) -> bool:
        return self._streams[index].query()

    def release_graphs(self) -> None:
        self._graphs.clear()


class Runner(Pipeline):
    """Two-slot asynchronous queue (src/runner.cc:17-68)."""

    def __init__(self, graph: bool = False):
        super().__init__(graph)
        self._head = 0
        self._queue: deque = deque()

    @property
    def head_index(self) -> int:
        return self._head

    def enqueue(self, input_callback, output_callback, input_id: int, output_id: int) -> result:
        if len(self._queue) == self.number_of_streams():
            return result.runner_queue_full
        will = self.will_output()
        r = input_callback()
        if r not in (None, result.success):
            return r
        r = self.compute(self._head)
        if r != result.success:
            return r
        if will:
            r = output_callback()
            if r not in (None, result.success):
                return r
        self._queue.append((self._head, input_id, output_id, will))
        self._head = (self._head + 1) % self.number_of_streams()
        return result.success

    def dequeue(self, callback) -> result:
        if not self._queue:
            return result.runner_queue_empty
        front, in_id, out_id, did = self._queue[0]
        if len(self._queue) < self.number_of_streams():
            if not self.is_synchronized(front):
                return result.runner_queue_none_available
        else:
            self.synchronize(front)
        self._queue.popleft()
        r = callback(in_id, out_id, did)
        return result.success if r in (None, True) else r

    def copy(self, dst, src) -> result:
        """Copy on the head slot's stream; a Duet operand resolves to its head slot
        (include/blade/runner.hh:29-47)."""
        if isinstance(dst, Duet):
            dst = dst[self._head]
        if isinstance(src, Duet):
            src = src.at(self._head)
        _copy(dst, src, self.stream(self._head))
        return result.success


def runner(cls=None, *, graph: bool = False):
    """Class decorator (python/blade/_runner/__init__.py:6-86).  The decorated
    class's ``__init__`` declares buffers and modules; the instance gains
    ``input``/``output``/``module`` namespaces, ``copy``, ``enqueue``, ``dequeue``
    and ``__call__(*transfer_in_args, *transfer_out_args)``."""

    def wrap(klass):
        class BasePipeline(klass):
            def __init__(self, *args, **kwargs):
                self.runner = Runner(graph=graph)
                self.input = SimpleNamespace()
                self.output = SimpleNamespace()
                self.module = SimpleNamespace()
                with _building(self.runner):
                    super().__init__(*args, **kwargs)

            def copy(self, dst, src):
                assert self.runner.copy(dst, src) == result.success

            def enqueue(self, input_callback, output_callback, input_id, output_id):
                return self.runner.enqueue(input_callback, output_callback, input_id, output_id)

            def dequeue(self, callback):
                return self.runner.dequeue(callback)

            def __call__(self, *args):
                if not hasattr(self, "transfer_in"):
                    raise AttributeError("The 'transfer_in' function is missing in the pipeline.")
                if not hasattr(self, "transfer_out"):
                    raise AttributeError("The 'transfer_out' function is missing in the pipeline.")
                for ns in (self.input, self.output):
                    for v in vars(ns).values():
                        if isinstance(v, Duet):
                            v.set(0)
                n_in = self.transfer_in.__code__.co_argcount - 1
                n_out = self.transfer_out.__code__.co_argcount - 1
                if len(args) != n_in + n_out:
                    raise ValueError(f"Expected {n_in + n_out} arguments, but got {len(args)}.")
                will = self.runner.will_output()
                self.runner._head = 0
                self.transfer_in(*args[:n_in])
                assert self.runner.compute(0) == result.success
                if will:
                    self.transfer_out(*args[n_in:])
                assert self.runner.synchronize(0) == result.success
                return will

            def synchronize(self):
                assert self.runner.synchronize(0) == result.success

        BasePipeline.__name__ = klass.__name__
        BasePipeline.__qualname__ = klass.__qualname__
        return BasePipeline

    if cls is not None:
        return wrap(cls)
    return wrap


def _sanitize(obj, index=0):
    """python/blade/_internal/__init__.py:81-100: a Duet stands for its slot."""
    if isinstance(obj, Duet):
        return obj[index]
    return obj


def module(name, config, input, it=None, ot=None, telescope=K.generic):
    """Instantiate a module and register it in the pipeline under construction
    (python/blade/_modules/__init__.py:105-248)."""
    if not isinstance(name, Constant):
        raise ValueError("Module name has to be a constant type (`bl.beamformer`, `bl.phasor`, etc).")
    if not isinstance(telescope, Constant):
        raise ValueError("Module telescope has to be a constant type (`bl.generic`, `bl.ata`, `bl.vla`, etc).")
    _name, _tel = name.value, telescope.value
    tels = sorted({t for (n, t) in REGISTRY if n == _name})
    if not tels:
        raise ModuleNotFoundError(f"Can't find specified module extension ({_name}).")
    if _tel not in tels:
        if tels == ["generic"]:
            raise AttributeError(f"The module '{_name}' only supports generic telescopes (telescope=bl.generic).")
        raise AttributeError(f"The module '{_name}' only supports these telescopes: {', '.join(tels)}.")
    cls, pairs = REGISTRY[(_name, _tel)]
    default_in, default_out = sorted(pairs)[0] if len(pairs) == 1 else ("cf32", "cf32")
    if _name == "detector":
        default_in, default_out = "cf32", "f32"
    if _name == "phasor":
        default_in, default_out = "f64", "cf32"
    if _name in ("beamform_detect", "modeh", "modeb"):
        default_in, default_out = "ci8", "f32"
    for label, v in (("input", it), ("output", ot)):
        if v is not None and not isinstance(v, Constant):
            raise ValueError(f"Module {label} data type has to be a constant type (`bl.cf32`, `bl.f32`, etc).")
    _it = it.value if it is not None else default_in
    _ot = ot.value if ot is not None else default_out
    ins = sorted({a for a, _ in pairs})
    if _it not in ins:
        raise AttributeError(f"The module '{_name}' only supports these input types: {', '.join(ins)}.")
    outs = sorted({b for a, b in pairs if a == _it})
    if _ot not in outs:
        raise AttributeError(
            f"The module '{_name}' with input '{_it}' only supports these output types: {', '.join(outs)}.")

    cfg_cls, in_cls = cls.config, cls.input
    if isinstance(config, cfg_cls):
        cfg = config
    elif isinstance(config, tuple):
        cfg = cfg_cls(*config)
    elif isinstance(config, dict):
        cfg = cfg_cls(**config)
    elif isinstance(config, int):
        cfg = cfg_cls(config)
    else:
        raise ValueError("Config should be a Tuple, Dict, or Int.")

    if isinstance(input, in_cls):
        inp = input
    elif isinstance(input, tuple):
        inp = in_cls(*tuple(_sanitize(x) for x in input))
    elif isinstance(input, dict):
        inp = in_cls(**{k: _sanitize(v) for k, v in input.items()})
    elif isinstance(input, (Vector, Duet)):
        inp = in_cls(_sanitize(input))
    else:
        raise ValueError("Input should be a Tuple, Dict, or Vector.")

    pipeline = _fetch_pipeline()
    if pipeline is not None:
        if pipeline.commited():
            raise RuntimeError("Can't connect new module after Pipeline is commited.")
        inst = cls(cfg, inp, pipeline.stream(), it=_it, ot=_ot)
        pipeline.add_module(inst)
    else:
        inst = cls(cfg, inp, None, it=_it, ot=_ot)
    return inst
