"""Python bindings of the twins-b200 C ABI (include/twinsb200.h), by ctypes.

The host-side mirror of the reference's `twins` interface: a topology (--k, --topo=leafspine,
--topo=graph --topofile --fail), a flow file (src,dst,flow_size,start_ns[,conn]), per-world
TCP parameters (--tcp --ecnK --queue --fin --spray --RngSeed --RngRun), batches of worlds
(--worlds), and the fct.csv columns established_ns / completed_ns (reference src/main.cu:139-1153).

The library is loaded from twins_b200/lib/libtwinsb200.so; there is no fallback: without the
native library (or without a CUDA device) every call raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libtwinsb200.so"
# the 25-run event-chain build (the reference's twins128)
LIB25_PATH = Path(__file__).resolve().parent / "lib" / "libtwinsb200_runs25.so"
# the build that records the enqueue trace (the reference's --qtrace)
LIB_TRACE_PATH = Path(__file__).resolve().parent / "lib" / "libtwinsb200_trace.so"

TB_OK, TB_WARN_INEXACT = 0, 1
TB_ERR = {-1: "bad argument", -2: "CUDA error", -3: "HBM budget exceeded", -4: "call out of order",
          -5: "device-side wait ran out"}
TOPO_FATTREE, TOPO_LEAFSPINE, TOPO_GRAPH = 0, 1, 2
TCP = {"newreno": 0, "dctcp": 1, "cubic": 2}
# tb_tx_record (the reference's RDMA TxRec layout)
TX_RECORD = np.dtype([("ts", "<i8"), ("node", "<i4"), ("dev", "<i4"), ("a", "<u4"), ("b", "<u4"), ("sport", "<u4"), ("seq", "<u4"),
                      ("size", "<u2"), ("kind", "u1"), ("ecn", "u1")], align=True)
assert TX_RECORD.itemsize == 40
COUNTERS = ["drops", "marks", "retx", "rto", "undecided_ties", "host_events", "switch_events",
            "ovf_active", "ovf_due", "ovf_ring", "ovf_ooo", "ovf_tx", "barrier_timeouts"]


class TwinsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{TB_ERR.get(code, code)}: {msg}")
        self.code = code


class _Topology(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("k", ctypes.c_int), ("leaves", ctypes.c_int), ("spines", ctypes.c_int),
                ("hpl", ctypes.c_int), ("n_hosts", ctypes.c_int), ("n_switches", ctypes.c_int), ("n_links", ctypes.c_int),
                ("link_a", ctypes.POINTER(ctypes.c_int)), ("link_b", ctypes.POINTER(ctypes.c_int)),
                ("n_fails", ctypes.c_int), ("fail_t_ns", ctypes.POINTER(ctypes.c_longlong)),
                ("fail_a", ctypes.POINTER(ctypes.c_int)), ("fail_b", ctypes.POINTER(ctypes.c_int)),
                ("fail_up", ctypes.POINTER(ctypes.c_int))]


class _TcpParams(ctypes.Structure):
    _fields_ = [("tcp", ctypes.c_int), ("ecn_k", ctypes.c_int), ("queue", ctypes.c_int), ("fin", ctypes.c_int),
                ("spray", ctypes.c_int), ("rng_seed", ctypes.c_uint), ("rng_run", ctypes.c_ulonglong)]


class _Stats(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_longlong), ("slots_run", ctypes.c_longlong), ("launches", ctypes.c_longlong),
                ("kernel_ms", ctypes.c_double), ("upload_ms", ctypes.c_double), ("packet_events", ctypes.c_ulonglong),
                ("host_events", ctypes.c_ulonglong), ("switch_events", ctypes.c_ulonglong),
                ("host_sender_events", ctypes.c_ulonglong), ("host_frames", ctypes.c_ulonglong),
                ("bytes_h2d", ctypes.c_ulonglong), ("bytes_d2h", ctypes.c_ulonglong),
                ("grid", ctypes.c_int), ("host_lanes", ctypes.c_int), ("warps_per_block", ctypes.c_int),
                ("stage_frames", ctypes.c_int), ("autotuned", ctypes.c_int), ("port_local", ctypes.c_int),
                ("graph_launches", ctypes.c_longlong)]


class _QRec(ctypes.Structure):
    _fields_ = [("ts", ctypes.c_longlong), ("node", ctypes.c_int), ("dev", ctypes.c_int), ("src", ctypes.c_int), ("dst", ctypes.c_int),
                ("sa", ctypes.c_uint), ("len", ctypes.c_ushort), ("qlen", ctypes.c_ushort), ("flags", ctypes.c_ubyte),
                ("pad", ctypes.c_ubyte * 3)]


class _ServeCaps(ctypes.Structure):
    _fields_ = [("worlds", ctypes.c_int), ("hosts", ctypes.c_int), ("switches", ctypes.c_int), ("ports", ctypes.c_int),
                ("connections", ctypes.c_int), ("messages", ctypes.c_int), ("sent_list_entries", ctypes.c_ulonglong),
                ("ooo_blocks", ctypes.c_ulonglong), ("active_per_host", ctypes.c_int), ("max_queue", ctypes.c_int),
                ("max_ports", ctypes.c_int), ("slots_per_launch", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_ulonglong)]


class _RequestInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("n_flows", ctypes.c_int), ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double), ("slot0", ctypes.c_longlong), ("slots", ctypes.c_longlong)]


class _ServeStats(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_longlong), ("slots_run", ctypes.c_longlong), ("admitted", ctypes.c_longlong),
                ("retired", ctypes.c_longlong), ("queued", ctypes.c_longlong), ("running", ctypes.c_longlong),
                ("kernel_ms", ctypes.c_double), ("packet_events", ctypes.c_ulonglong), ("hbm_bytes", ctypes.c_ulonglong),
                ("host_lanes", ctypes.c_int), ("stage_frames", ctypes.c_int), ("grid", ctypes.c_int)]


# every entry point of include/twinsb200.h: (name, restype, argtypes)
_P = ctypes.POINTER
ENTRY_POINTS = [
    ("tb_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.c_ulonglong, _P(ctypes.c_void_p)]),
    ("tb_ctx_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("tb_last_error", ctypes.c_char_p, []),
    ("tb_world_add_tcp", ctypes.c_int, [ctypes.c_void_p, _P(_Topology), ctypes.c_int, _P(ctypes.c_int), _P(ctypes.c_int),
                                        _P(ctypes.c_longlong), _P(ctypes.c_longlong), _P(ctypes.c_longlong),
                                        _P(ctypes.c_uint), _P(ctypes.c_uint), _P(_TcpParams), _P(ctypes.c_int)]),
    ("tb_world_add_rdma", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, _P(ctypes.c_int), _P(ctypes.c_int),
                                         _P(ctypes.c_longlong), _P(ctypes.c_longlong), ctypes.c_ulonglong, ctypes.c_longlong,
                                         _P(ctypes.c_int)]),
    ("tb_rdma_results", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_longlong), _P(ctypes.c_longlong)]),
    ("tb_rdma_set_queue_cap", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("tb_rdma_set_txtrace", ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong]),
    ("tb_rdma_txtrace", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, _P(ctypes.c_longlong), _P(ctypes.c_longlong)]),
    ("tb_prepare", ctypes.c_int, [ctypes.c_void_p]),
    ("tb_reset", ctypes.c_int, [ctypes.c_void_p]),
    ("tb_run", ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    ("tb_results", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_longlong), _P(ctypes.c_longlong)]),
    ("tb_counters", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_ulonglong), ctypes.c_int]),
    ("tb_hashes", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_uint), _P(ctypes.c_uint)]),
    ("tb_get_stats", ctypes.c_int, [ctypes.c_void_p, _P(_Stats)]),
    ("tb_set_launch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    ("tb_set_launch_shape", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("tb_set_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("tb_set_port_local", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("tb_set_free_batches", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("tb_abi_sizes", ctypes.c_int, [_P(ctypes.c_ulonglong), ctypes.c_int]),
    ("tb_has_qtrace", ctypes.c_int, []),
    ("tb_set_qtrace", ctypes.c_int, [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_longlong]),
    ("tb_qtrace", ctypes.c_int, [ctypes.c_void_p, _P(_QRec), ctypes.c_ulonglong, _P(ctypes.c_ulonglong)]),
    ("tb_server_create", ctypes.c_int, [ctypes.c_int, _P(_ServeCaps), _P(ctypes.c_void_p)]),
    ("tb_server_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("tb_server_submit_tcp", ctypes.c_int, [ctypes.c_void_p, _P(_Topology), ctypes.c_int, _P(ctypes.c_int), _P(ctypes.c_int),
                                            _P(ctypes.c_longlong), _P(ctypes.c_longlong), _P(ctypes.c_longlong), _P(_TcpParams),
                                            _P(ctypes.c_longlong)]),
    ("tb_server_step", ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_int)]),
    ("tb_server_start", ctypes.c_int, [ctypes.c_void_p]),
    ("tb_server_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double]),
    ("tb_server_results", ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, _P(ctypes.c_longlong), _P(ctypes.c_longlong),
                                         _P(ctypes.c_ulonglong), ctypes.c_int, _P(_RequestInfo)]),
    ("tb_server_release", ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    ("tb_server_stats", ctypes.c_int, [ctypes.c_void_p, _P(_ServeStats)]),
    ("tb_run_static", ctypes.c_int, [ctypes.c_int, _P(_Topology), ctypes.c_int, _P(ctypes.c_int), _P(ctypes.c_int),
                                     _P(ctypes.c_longlong), _P(ctypes.c_longlong), _P(ctypes.c_longlong),
                                     _P(_TcpParams), ctypes.c_longlong, _P(ctypes.c_longlong), _P(ctypes.c_longlong)]),
]

_lib = None


def load_library(path: Optional[os.PathLike] = None) -> ctypes.CDLL:
    """Loads libtwinsb200.so (built by twins_b200.build); raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: run `python -m twins_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    for name, res, args in ENTRY_POINTS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    sizes = (ctypes.c_ulonglong * 8)()
    lib.tb_abi_sizes(sizes, 8)
    want = [ctypes.sizeof(_Topology), ctypes.sizeof(_TcpParams), ctypes.sizeof(_Stats), ctypes.sizeof(_ServeCaps),
            ctypes.sizeof(_RequestInfo), ctypes.sizeof(_ServeStats), ctypes.sizeof(_QRec), TX_RECORD.itemsize]
    if list(sizes) != want:
        raise RuntimeError(f"{p}: struct sizes {list(sizes)} differ from these bindings' {want}: rebuild")
    if path is None:
        _lib = lib
    return lib


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


# ------------------------------------------------------------------ inputs
@dataclass
class Topology:
    """A world's topology: FatTree(k), leaf-spine(leaves, spines, hpl) or a topology file."""
    kind: int = TOPO_FATTREE
    k: int = 4
    leaves: int = 16
    spines: int = 8
    hpl: int = 16
    n_hosts: int = 0
    n_switches: int = 0
    links: list = field(default_factory=list)   # [(a, b)]: host h -> h, switch j -> -1 - j
    fails: list = field(default_factory=list)   # [(t_ns, sA, sB, up)]

    @staticmethod
    def fattree(k: int) -> "Topology":
        return Topology(kind=TOPO_FATTREE, k=k)

    @staticmethod
    def leafspine(leaves: int, spines: int, hpl: int) -> "Topology":
        return Topology(kind=TOPO_LEAFSPINE, leaves=leaves, spines=spines, hpl=hpl)

    @staticmethod
    def from_file(path: os.PathLike, fail: str = "") -> "Topology":
        """A topology file (workloads/topo.py format: hosts H, switches S, link A B lines) and a
        --fail spec T:sA:sB[:up],... (reference src/main.cu:227-252, 373-465)."""
        t = Topology(kind=TOPO_GRAPH)
        toks = Path(path).read_text().split()
        node = lambda x: int(x[1:]) if x[0] == "h" else -1 - int(x[1:])
        i = 0
        while i < len(toks):
            key = toks[i]
            if key == "hosts":
                t.n_hosts = int(toks[i + 1]); i += 2
            elif key == "switches":
                t.n_switches = int(toks[i + 1]); i += 2
            elif key == "link":
                t.links.append((node(toks[i + 1]), node(toks[i + 2]))); i += 3
            else:
                i += 1
        for item in filter(None, fail.split(",")):
            v = item.split(":")
            if len(v) < 3:
                raise ValueError("--fail: T:sA:sB[:up]")
            t.fails.append((int(v[0]), int(v[1][1:]), int(v[2][1:]), len(v) > 3 and v[3] == "up"))
        return t

    @staticmethod
    def from_args(args: Sequence[str], base: Optional[Path] = None) -> "Topology":
        """From the reference's topology flags (--k=, --topo=, --leaves= ...)."""
        kv = dict(a[2:].split("=", 1) for a in args if a.startswith("--") and "=" in a)
        topo = kv.get("topo", "fattree")
        if topo == "graph":
            f = Path(kv["topofile"])
            if base is not None and not f.is_absolute():
                f = base / f
            return Topology.from_file(f, kv.get("fail", ""))
        if topo == "leafspine":
            return Topology.leafspine(int(kv.get("leaves", 16)), int(kv.get("spines", 8)), int(kv.get("hpl", 16)))
        return Topology.fattree(int(kv.get("k", 4)))

    @property
    def hosts(self) -> int:
        if self.kind == TOPO_GRAPH:
            return self.n_hosts
        if self.kind == TOPO_LEAFSPINE:
            return self.leaves * self.hpl
        return self.k ** 3 // 4

    def _c(self):
        keep = []
        t = _Topology(self.kind, self.k, self.leaves, self.spines, self.hpl, self.n_hosts, self.n_switches, len(self.links))
        if self.links:
            la = np.array([a for a, _ in self.links], dtype=np.int32)
            lb = np.array([b for _, b in self.links], dtype=np.int32)
            keep += [la, lb]
            t.link_a, t.link_b = _ptr(la, ctypes.c_int), _ptr(lb, ctypes.c_int)
        if self.fails:
            ft = np.array([f[0] for f in self.fails], dtype=np.int64)
            fa = np.array([f[1] for f in self.fails], dtype=np.int32)
            fb = np.array([f[2] for f in self.fails], dtype=np.int32)
            fu = np.array([int(bool(f[3])) for f in self.fails], dtype=np.int32)
            keep += [ft, fa, fb, fu]
            t.n_fails = len(self.fails)
            t.fail_t_ns, t.fail_a = _ptr(ft, ctypes.c_longlong), _ptr(fa, ctypes.c_int)
            t.fail_b, t.fail_up = _ptr(fb, ctypes.c_int), _ptr(fu, ctypes.c_int)
        return t, keep


@dataclass
class Flows:
    """Rows of a flow file: src, dst, size (bytes), start_ns, conn (-1: own connection)."""
    src: np.ndarray
    dst: np.ndarray
    size: np.ndarray
    start_ns: np.ndarray
    conn: np.ndarray

    def __len__(self) -> int:
        return len(self.src)

    @staticmethod
    def from_arrays(src, dst, size, start_ns, conn=None) -> "Flows":
        n = len(src)
        return Flows(np.ascontiguousarray(src, dtype=np.int32), np.ascontiguousarray(dst, dtype=np.int32),
                     np.ascontiguousarray(size, dtype=np.int64), np.ascontiguousarray(start_ns, dtype=np.int64),
                     np.ascontiguousarray(conn if conn is not None else np.full(n, -1), dtype=np.int64))

    @staticmethod
    def load(path: os.PathLike, hosts: int) -> "Flows":
        """src,dst,flow_size,start_ns[,conn] or node,flow_size,start_ns (host i with i + H/2);
        lines not starting with a digit are skipped (reference src/main.cu:110-137)."""
        src, dst, size, start, conn = [], [], [], [], []
        for line in Path(path).read_text().splitlines():
            if not line or not line[0].isdigit():
                continue
            v = [int(x) for x in line.split(",")]
            if len(v) == 3:
                src.append(v[0]); dst.append((v[0] + hosts // 2) % hosts); size.append(v[1]); start.append(v[2]); conn.append(-1)
            elif len(v) >= 4:
                src.append(v[0]); dst.append(v[1]); size.append(v[2]); start.append(v[3])
                conn.append(v[4] if len(v) >= 5 else -1)
        return Flows.from_arrays(src, dst, size, start, conn)

    def write_csv(self, path: os.PathLike) -> None:
        has_conn = bool((self.conn >= 0).any())
        with open(path, "w") as f:
            f.write("src,dst,flow_size,start_ns" + (",conn" if has_conn else "") + "\n")
            for i in range(len(self)):
                row = f"{self.src[i]},{self.dst[i]},{self.size[i]},{self.start_ns[i]}"
                f.write(row + (f",{self.conn[i]}" if has_conn else "") + "\n")


@dataclass
class TcpParams:
    tcp: str = "dctcp"
    ecn_k: int = 30
    queue: int = 200
    fin: bool = False
    spray: bool = False
    rng_seed: int = 1
    rng_run: int = 1

    @staticmethod
    def from_args(args: Sequence[str], tcp: str = "dctcp") -> "TcpParams":
        kv = dict(a[2:].split("=", 1) for a in args if a.startswith("--") and "=" in a)
        return TcpParams(tcp=kv.get("tcp", tcp), ecn_k=int(kv.get("ecnK", 30)), queue=int(kv.get("queue", 200)),
                         fin=kv.get("fin", "0") != "0", spray=kv.get("spray", "0") != "0",
                         rng_seed=int(kv.get("RngSeed", 1)), rng_run=int(kv.get("RngRun", 1)))

    def _c(self):
        return _TcpParams(TCP[self.tcp], self.ecn_k, self.queue, int(self.fin), int(self.spray), self.rng_seed, self.rng_run)


# ------------------------------------------------------------------ the simulator
class Simulator:
    """A batch of worlds on one GPU: add worlds, run, read results (tb_* of the C ABI)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, host_lanes: Optional[int] = None, grid: int = 0,
                 stage_frames: int = 192, chain_runs: int = 9, port_local: bool = False, free_batches: bool = True):
        """host_lanes None: the launch shape is autotuned per launch; else that fixed shape.
        chain_runs 25: the 25-run event-chain build (the reference's twins128).
        free_batches False: a batch's worlds share one barrier per slot (else each has its own)."""
        if chain_runs not in (9, 25):
            raise ValueError("chain_runs is 9 or 25")
        self.lib = load_library(LIB25_PATH if chain_runs == 25 else None)
        self.ctx = ctypes.c_void_p()
        self._check(self.lib.tb_ctx_create(device, hbm_budget_bytes, ctypes.byref(self.ctx)))
        if host_lanes is not None:
            self._check(self.lib.tb_set_launch_shape(self.ctx, host_lanes, stage_frames, grid))
            self._check(self.lib.tb_set_port_local(self.ctx, int(port_local)))
        if not free_batches:
            self._check(self.lib.tb_set_free_batches(self.ctx, 0))
        self.sizes: list[int] = []
        self.last_status = TB_OK

    def _check(self, r: int) -> int:
        if r < 0:
            raise TwinsError(r, self.lib.tb_last_error().decode())
        return r

    def add_world(self, topo: Topology, flows: Flows, params: TcpParams,
                  hash_data: Optional[np.ndarray] = None, hash_ack: Optional[np.ndarray] = None) -> int:
        t, keep = topo._c()
        p = params._c()
        wid = ctypes.c_int()
        hd = ha = None
        if hash_data is not None:
            hd = np.ascontiguousarray(hash_data, dtype=np.uint32)
            ha = np.ascontiguousarray(hash_ack, dtype=np.uint32)
        self._check(self.lib.tb_world_add_tcp(
            self.ctx, ctypes.byref(t), len(flows), _ptr(flows.src, ctypes.c_int), _ptr(flows.dst, ctypes.c_int),
            _ptr(flows.size, ctypes.c_longlong), _ptr(flows.start_ns, ctypes.c_longlong), _ptr(flows.conn, ctypes.c_longlong),
            _ptr(hd, ctypes.c_uint) if hd is not None else None, _ptr(ha, ctypes.c_uint) if ha is not None else None,
            ctypes.byref(p), ctypes.byref(wid)))
        del keep
        self.sizes.append(len(flows))
        return wid.value

    def add_rdma_world(self, config: str, topology: str, flows: Flows, link_bps: int = 100_000_000_000,
                       link_delay_ns: int = 1000) -> int:
        """An RDMA world (tb_world_add_rdma): the HPCC config's "KEY VALUE" text, a TwiNS topology
        text (hosts / switches / link), the flows (src, dst, size, start_ns; conn unused)."""
        wid = ctypes.c_int()
        self._check(self.lib.tb_world_add_rdma(
            self.ctx, config.encode(), topology.encode(), len(flows), _ptr(flows.src, ctypes.c_int), _ptr(flows.dst, ctypes.c_int),
            _ptr(flows.size, ctypes.c_longlong), _ptr(flows.start_ns, ctypes.c_longlong), int(link_bps), int(link_delay_ns),
            ctypes.byref(wid)))
        self.sizes.append(len(flows))
        return wid.value

    def set_rdma_queue_cap(self, frames: int) -> None:
        """Frames a switch port's data queue holds (the reference's --q3cap; before the first run)."""
        self._check(self.lib.tb_rdma_set_queue_cap(self.ctx, frames))

    def set_rdma_txtrace(self, cap: int, from_ns: int = 0, until_ns: int = 1 << 62) -> None:
        """Keep up to `cap` transmission records (the reference's --txtrace; one world, before the run)."""
        self._check(self.lib.tb_rdma_set_txtrace(self.ctx, cap, from_ns, until_ns))

    def rdma_txtrace(self) -> tuple[list[str], int]:
        """The run's transmissions as the reference's --txtrace lines ("ns node dev kind src dst sport
        seq bytes ecn", sorted by ns, node, dev), and how many there were in the window."""
        n, total = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.tb_rdma_txtrace(self.ctx, None, 0, ctypes.byref(n), ctypes.byref(total)))
        rec = np.zeros(total.value, dtype=TX_RECORD)
        self._check(self.lib.tb_rdma_txtrace(self.ctx, rec.ctypes.data_as(ctypes.c_void_p), len(rec), ctypes.byref(n), ctypes.byref(total)))
        lines = [f"{r['ts']} {r['node']} {r['dev']} {'DANPR'[r['kind']]} {r['a']} {r['b']} {r['sport']} {r['seq']} {r['size']} {r['ecn']}"
                 for r in rec[:n.value]]
        return lines, total.value

    def rdma_results(self, world: int) -> tuple[np.ndarray, np.ndarray]:
        """(start_ns, fct_ns) per flow of an RDMA world; fct -1: not done."""
        n = self.sizes[world]
        start = np.empty(n, dtype=np.int64)
        fct = np.empty(n, dtype=np.int64)
        self._check(self.lib.tb_rdma_results(self.ctx, world, _ptr(start, ctypes.c_longlong), _ptr(fct, ctypes.c_longlong)))
        return start, fct

    def rdma_counters(self, world: int = 0) -> list[int]:
        """The run's 40 RDMA counters in the reference's order."""
        out = np.zeros(40, dtype=np.uint64)
        self._check(self.lib.tb_counters(self.ctx, world, _ptr(out, ctypes.c_ulonglong), 40))
        return [int(x) for x in out]

    def prepare(self) -> None:
        self._check(self.lib.tb_prepare(self.ctx))

    def reset(self) -> None:
        self._check(self.lib.tb_reset(self.ctx))

    def run(self, max_slots: int = 0) -> int:
        self.last_status = self._check(self.lib.tb_run(self.ctx, max_slots))
        return self.last_status

    def results(self, world: int) -> tuple[np.ndarray, np.ndarray]:
        n = self.sizes[world]
        est = np.empty(n, dtype=np.int64)
        done = np.empty(n, dtype=np.int64)
        self._check(self.lib.tb_results(self.ctx, world, _ptr(est, ctypes.c_longlong), _ptr(done, ctypes.c_longlong)))
        return est, done

    def counters(self, world: int) -> dict:
        out = np.zeros(16, dtype=np.uint64)
        self._check(self.lib.tb_counters(self.ctx, world, _ptr(out, ctypes.c_ulonglong), 16))
        return {name: int(out[i]) for i, name in enumerate(COUNTERS)}

    def hashes(self, world: int) -> tuple[np.ndarray, np.ndarray]:
        n = self.sizes[world]
        hd = np.empty(n, dtype=np.uint32)
        ha = np.empty(n, dtype=np.uint32)
        self._check(self.lib.tb_hashes(self.ctx, world, _ptr(hd, ctypes.c_uint), _ptr(ha, ctypes.c_uint)))
        return hd, ha

    def stats(self) -> dict:
        s = _Stats()
        self._check(self.lib.tb_get_stats(self.ctx, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in _Stats._fields_}

    def close(self) -> None:
        if self.ctx:
            self.lib.tb_ctx_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


RDMA_COUNTERS_LINE = ("drops {0} marks {1} pauses {2} resumes {3} nacks {11} | undecided ties {8}, on lost tails {9} | "
                      "overflows: tx {4} queue {5} ackq {6} qps {7} due {12} | acks for done QPs {10}")


def rdma_counters_line(ev) -> str:
    """The reference's counters line of twins-rdma (src/rdma/rmain.cu:2239-2261)."""
    return RDMA_COUNTERS_LINE.format(*ev)


def run_rdma_world(config: str, topology: str, flows: Flows, link_bps: int = 100_000_000_000, link_delay_ns: int = 1000,
                   max_slots: int = 0, device: int = 0, queue_cap: int = 0):
    """One RDMA world: (start_ns, fct_ns, counters, stats, status)."""
    with Simulator(device=device) as sim:
        if queue_cap:
            sim.set_rdma_queue_cap(queue_cap)
        w = sim.add_rdma_world(config, topology, flows, link_bps, link_delay_ns)
        status = sim.run(max_slots)
        start, fct = sim.rdma_results(w)
        return start, fct, sim.rdma_counters(w), sim.stats(), status


def run_world(topo: Topology, flows: Flows, params: TcpParams, max_slots: int = 0, **kw):
    """One world: (established_ns, completed_ns, counters, stats)."""
    with Simulator(**kw) as sim:
        w = sim.add_world(topo, flows, params)
        sim.run(max_slots)
        est, done = sim.results(w)
        return est, done, sim.counters(w), sim.stats()


def run_world_static(topo: Topology, flows: Flows, params: TcpParams, max_slots: int = 0, device: int = 0):
    """One world through tb_run_static, which allocates no device memory (for callers that may
    not allocate: the world's device state lives in the library's fixed area). Returns
    (established_ns, completed_ns, status)."""
    lib = load_library()
    t, keep = topo._c()
    p = params._c()
    n = len(flows)
    est = np.empty(n, dtype=np.int64)
    done = np.empty(n, dtype=np.int64)
    r = lib.tb_run_static(device, ctypes.byref(t), n, _ptr(flows.src, ctypes.c_int), _ptr(flows.dst, ctypes.c_int),
                          _ptr(flows.size, ctypes.c_longlong), _ptr(flows.start_ns, ctypes.c_longlong),
                          _ptr(flows.conn, ctypes.c_longlong), ctypes.byref(p), max_slots,
                          _ptr(est, ctypes.c_longlong), _ptr(done, ctypes.c_longlong))
    del keep
    if r < 0:
        raise TwinsError(r, lib.tb_last_error().decode())
    return est, done, r


# ------------------------------------------------------------------ serving
class Server:
    """Continuous batching of simulation requests on one GPU (tb_server_* of the C ABI): requests
    join the running batch between launches and each runs exactly as it would alone."""

    def __init__(self, device: int = 0, worlds: int = 64, hosts: int = 8192, switches: int = 2048, ports: int = 32768,
                 connections: int = 1 << 18, messages: int = 1 << 18, sent_list_entries: int = 1 << 27, ooo_blocks: int = 1 << 25,
                 active_per_host: int = 256, max_queue: int = 400, max_ports: int = 32, slots_per_launch: int = 256,
                 hbm_budget_bytes: int = 0):
        self.lib = load_library()
        caps = _ServeCaps(worlds, hosts, switches, ports, connections, messages, sent_list_entries, ooo_blocks, active_per_host,
                          max_queue, max_ports, slots_per_launch, hbm_budget_bytes)
        self.srv = ctypes.c_void_p()
        self._check(self.lib.tb_server_create(device, ctypes.byref(caps), ctypes.byref(self.srv)))
        self.sizes: dict[int, int] = {}

    def _check(self, r: int) -> int:
        if r < 0:
            raise TwinsError(r, self.lib.tb_last_error().decode())
        return r

    def submit(self, topo: Topology, flows: Flows, params: TcpParams) -> int:
        t, keep = topo._c()
        p = params._c()
        rid = ctypes.c_longlong()
        self._check(self.lib.tb_server_submit_tcp(
            self.srv, ctypes.byref(t), len(flows), _ptr(flows.src, ctypes.c_int), _ptr(flows.dst, ctypes.c_int),
            _ptr(flows.size, ctypes.c_longlong), _ptr(flows.start_ns, ctypes.c_longlong), _ptr(flows.conn, ctypes.c_longlong),
            ctypes.byref(p), ctypes.byref(rid)))
        del keep
        self.sizes[rid.value] = len(flows)
        return rid.value

    def step(self) -> int:
        n = ctypes.c_int()
        self._check(self.lib.tb_server_step(self.srv, ctypes.byref(n)))
        return n.value

    def start(self) -> None:
        self._check(self.lib.tb_server_start(self.srv))

    def wait(self, request: int, timeout_s: float = 0.0) -> None:
        self._check(self.lib.tb_server_wait(self.srv, request, timeout_s))

    def info(self, request: int) -> dict:
        i = _RequestInfo()
        self._check(self.lib.tb_server_results(self.srv, request, None, None, None, 0, ctypes.byref(i)))
        return {name: getattr(i, name) for name, _ in _RequestInfo._fields_}

    def results(self, request: int) -> tuple[np.ndarray, np.ndarray, dict]:
        n = self.sizes[request]
        est = np.empty(n, dtype=np.int64)
        done = np.empty(n, dtype=np.int64)
        ctr = np.zeros(16, dtype=np.uint64)
        self._check(self.lib.tb_server_results(self.srv, request, _ptr(est, ctypes.c_longlong), _ptr(done, ctypes.c_longlong),
                                               _ptr(ctr, ctypes.c_ulonglong), 16, None))
        return est, done, {name: int(ctr[i]) for i, name in enumerate(COUNTERS)}

    def release(self, request: int) -> None:
        self._check(self.lib.tb_server_release(self.srv, request))
        self.sizes.pop(request, None)

    def stats(self) -> dict:
        s = _ServeStats()
        self._check(self.lib.tb_server_stats(self.srv, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in _ServeStats._fields_}

    def close(self) -> None:
        if self.srv:
            self.lib.tb_server_destroy(self.srv)
            self.srv = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
