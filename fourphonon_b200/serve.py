"""Serving loop: a stream of 3ph+4ph RTA solves on one GPU.

Requests (a Solve and a temperature) arrive over time.  They wait in a FIFO
until a slot is free and their device footprint fits the HBM budget, then
their inputs stay on the device while the server's ticks run.  Every tick is
one launch of the multi-solve kernel over a share of each running solve's
work items (fp4_server_tick), so solves that arrive while others run share
the GPU with them from their first tick on (continuous batching).  A finished
solve's rates and kappa are collected and its slot and memory are freed.

`run_stream` replays a list of (arrival time, solve, T) on the wall clock and
reports each request's latency (arrival to result) with the p50/p99 latency
and the solves/s of the whole stream.
"""
from __future__ import annotations

import ctypes as ct
import json
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .abi import FP4Error, _p

_SIGS = False


def _lib():
    global _SIGS
    lib = abi.load()
    if not _SIGS:
        lib.fp4_server_last_error.restype = ct.c_char_p
        lib.fp4_server_last_error.argtypes = [ct.c_void_p]
        lib.fp4_server_footprint.restype = ct.c_int64
        lib.fp4_server_footprint.argtypes = [ct.c_int32, ct.c_int32, ct.c_void_p, ct.c_int32, ct.c_int32, ct.c_int32]
        _SIGS = True
    return lib


def footprint(s) -> int:
    """Device bytes a solve holds while it is resident in a slot."""
    ng = np.ascontiguousarray(s.ngrid, np.int32)
    return int(_lib().fp4_server_footprint(s.nb, s.nlist, _p(ng), s.ifc3.ntri, s.ifc4.ntri, s.sym.nsymm_rot))


class Server:
    """One fp4_server: slots, work queues and the captured tick graph."""

    def __init__(self, device=0, precision=abi.FP4_PREC_MIXED, max_slots=16, max_bands=12, hbm_budget=16 << 30):
        self.lib = _lib()
        h = ct.c_void_p()
        rc = self.lib.fp4_server_create(ct.byref(h), device, precision, max_slots, max_bands, ct.c_int64(hbm_budget))
        if rc != 0:
            msg = self.lib.fp4_server_last_error(h).decode() if h else "fp4_server_create failed"
            if h:
                self.lib.fp4_server_destroy(h)
            raise FP4Error(rc, msg)
        self.h = h
        self.max_slots = max_slots
        self._ctx = abi.Context.__new__(abi.Context)  # only for globals_of / array marshalling
        self._ctx._keep = []
        self.requests = {}

    def close(self):
        if self.h:
            self.lib.fp4_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, rc):
        return FP4Error(rc, self.lib.fp4_server_last_error(self.h).decode())

    def admit(self, s, T):
        """Load solve `s` at temperature T into a free slot; returns the slot,
        or None when no slot or budget is free right now."""
        g = abi.Context.globals_of(self._ctx, s, T)
        e, v, z, lst, ijk = abi.Context._arrays(s)
        f3 = abi.Context._ifc(s.ifc3)
        f4 = abi.Context._ifc(s.ifc4)
        w = s.wedge
        nsr = s.sym.nsymm_rot
        nequi = np.ascontiguousarray(w.nequi, np.int32)
        allequi = np.ascontiguousarray(w.allequi, np.int32)
        crot = np.ascontiguousarray(np.transpose(s.sym.crotations, (0, 2, 1))).ravel()
        slot = ct.c_int32(-1)
        rc = self.lib.fp4_server_admit(self.h, ct.byref(g), _p(e), _p(v), _p(z), s.nlist, _p(lst), _p(ijk),
                                       s.ifc3.ntri, *[_p(x) for x in f3], s.ifc4.ntri, *[_p(x) for x in f4], nsr,
                                       _p(nequi), _p(allequi), _p(crot), ct.c_double(s.volume), ct.byref(slot))
        if rc == abi.FP4_E_STATE:
            return None
        if rc != 0:
            raise self._err(rc)
        self.requests[slot.value] = s
        return slot.value

    def tick(self, max_items):
        """One launch over up to max_items work items; returns the finished slots."""
        fin = (ct.c_int32 * self.max_slots)()
        nf = ct.c_int32(0)
        rc = self.lib.fp4_server_tick(self.h, ct.c_int64(int(max_items)), fin, ct.byref(nf))
        if rc != 0:
            raise self._err(rc)
        return [fin[i] for i in range(nf.value)]

    def collect(self, slot):
        s = self.requests.pop(slot)
        nm = s.nmodes
        out = {k: np.zeros(nm) for k in ("rate3_plus", "rate3_minus", "rate4_pp", "rate4_pm", "rate4_mm")}
        kb = np.zeros(9 * s.nb)
        k = np.zeros(9)
        n = ct.c_int64(0)
        rc = self.lib.fp4_server_collect(self.h, slot, *[_p(out[x]) for x in ("rate3_plus", "rate3_minus", "rate4_pp",
                                                                               "rate4_pm", "rate4_mm")],
                                         _p(kb), _p(k), ct.byref(n))
        if rc != 0:
            raise self._err(rc)
        out["kappa_branch"] = kb.reshape(s.nb, 3, 3).transpose(0, 2, 1)  # [b][d1][d2]
        out["kappa"] = k.reshape(3, 3).T
        out["n_processes"] = n.value
        return out

    def status(self):
        r = ct.c_int32()
        d = ct.c_int32()
        b = ct.c_int64()
        ms = ct.c_double()
        t = ct.c_int64()
        self.lib.fp4_server_status(self.h, ct.byref(r), ct.byref(d), ct.byref(b), ct.byref(ms), ct.byref(t))
        return dict(running=r.value, done=d.value, bytes_in_use=b.value, last_tick_ms=ms.value, ticks=t.value)


@dataclass
class Request:
    arrival: float  # seconds after the start of the stream
    solve: object
    T: float
    tag: object = None
    admitted: float = -1.0
    finished: float = -1.0
    result: dict = field(default_factory=dict)

    @property
    def latency(self):
        return self.finished - self.arrival


def run_stream(server: Server, requests, tick_items=200_000, clock=time.perf_counter, sleep=time.sleep,
               target_tick_ms=None, max_tick_items=1 << 22, metrics=None):
    """Serve `requests` (sorted by arrival) on the wall clock; returns them with
    admission/finish times and results, plus a summary dict.

    With target_tick_ms, the number of work items per tick follows the last
    tick's device time so that a tick lasts about that long: long enough to
    hide the per-tick host work, short enough to admit new requests often.

    metrics: a writable text stream that receives one JSON line per finished
    request (tag, arrival, admission and finish times, latency, processes) as
    it finishes, and one line with the summary at the end."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    waiting = []
    running = {}
    nxt = 0
    t0 = clock()
    ticks = 0
    items = int(tick_items)
    t_admit = t_tick = t_collect = 0.0
    while nxt < len(reqs) or waiting or running:
        now = clock() - t0
        while nxt < len(reqs) and reqs[nxt].arrival <= now:
            waiting.append(reqs[nxt])
            nxt += 1
        while waiting:  # FIFO admission while slots and budget allow
            r = waiting[0]
            ta = clock()
            slot = server.admit(r.solve, r.T)
            t_admit += clock() - ta
            if slot is None:
                break
            r.admitted = clock() - t0
            running[slot] = r
            waiting.pop(0)
        if running:
            tt = clock()
            done = server.tick(items)
            t_tick += clock() - tt
            for slot in done:
                r = running.pop(slot)
                tc = clock()
                r.result = server.collect(slot)
                t_collect += clock() - tc
                r.finished = clock() - t0
                if metrics is not None:
                    _emit(metrics, event="request", tag=_plain(r.tag), arrival_s=r.arrival, admitted_s=r.admitted,
                          finished_s=r.finished, latency_ms=1e3 * r.latency,
                          processes=int(r.result.get("n_processes", 0)))
            ticks += 1
            if target_tick_ms:
                ms = server.status()["last_tick_ms"] if hasattr(server, "status") else 0.0
                if ms > 0:
                    items = int(min(max_tick_items, max(4096, items * target_tick_ms / ms)))
        elif nxt < len(reqs):
            sleep(max(0.0, reqs[nxt].arrival - (clock() - t0)))
    wall = clock() - t0
    lat = np.array([r.latency for r in reqs])
    summary = dict(requests=len(reqs), wall_s=wall, solves_per_s=len(reqs) / wall if wall > 0 else 0.0,
                   p50_ms=1e3 * float(np.percentile(lat, 50)), p99_ms=1e3 * float(np.percentile(lat, 99)),
                   mean_ms=1e3 * float(lat.mean()), ticks=ticks,
                   processes=int(sum(r.result.get("n_processes", 0) for r in reqs)),
                   host_s={"admit": t_admit, "tick": t_tick, "collect": t_collect})
    summary["processes_per_s"] = summary["processes"] / wall if wall > 0 else 0.0
    if metrics is not None:
        _emit(metrics, event="summary", **summary)
    return reqs, summary


def _plain(x):
    return x if isinstance(x, (int, float, str, bool)) or x is None else str(x)


def _emit(stream, **fields):
    stream.write(json.dumps(fields) + "\n")
    stream.flush()
