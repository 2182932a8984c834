"""Shared by the RDMA rule tests: the C shim over twins_b200/csrc/tr_*.cuh (tests/rdma_cc.cpp built
with g++, or tests/rdma_cc_gpu.cu built with nvcc for sm_100a, each function then run on the
device), its ctypes structures and signatures, and the reference's known answers
(tests/golden/rdma_kat.json.gz, made by tests/golden/make_rdma_kat.py)."""
import ctypes as C
import gzip
import json
import struct
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "twins_b200" / "csrc"
SHIM = ROOT / "tests" / "rdma_cc.cpp"
SHIM_GPU = ROOT / "tests" / "rdma_cc_gpu.cu"
KAT = ROOT / "tests" / "golden" / "rdma_kat.json.gz"

U64, U32, U8 = C.c_uint64, C.c_uint32, C.c_uint8


class QpRate(C.Structure):
    _fields_ = [("rate", U64), ("max_rate", U64), ("target", U64), ("snd_nxt", U64), ("base_rtt", U64), ("win", U32),
                ("alpha_cnp", U8), ("dec_cnp", U8), ("first_cnp", U8), ("rp_stage", U32), ("alpha", C.c_double),
                ("last_update_seq", U32), ("inc_stage", C.c_int32), ("cur_rate", U64), ("u", C.c_double), ("hop", U64 * 5),
                ("high_seq", U32), ("ecn_cnt", U32), ("batch", U32), ("ca_state", U32)]


class CcParams(C.Structure):
    _fields_ = [("g", C.c_double), ("rate_first_cnp", C.c_double), ("clamp", C.c_int), ("rpg_threshold", U32), ("rai", U64),
                ("rhai", U64), ("min_rate", U64), ("dctcp_rai", U64), ("u_target", C.c_double), ("mi_thresh", U32),
                ("sample_feedback", C.c_int), ("int_multi", U32), ("mtu", U32)]


class NicParams(C.Structure):
    _fields_ = [("mtu", U32), ("ack_interval", U32), ("chunk", U32), ("nack_interval", C.c_int64), ("seq_extra", U32), ("int_size", C.c_int),
                ("var_win", C.c_int), ("ack_high_prio", C.c_int), ("cc", C.c_int), ("fast_react", C.c_int), ("ns336", C.c_int)]


class QpSend(C.Structure):
    _fields_ = [("size", U64), ("snd_una", U64), ("next_avail", C.c_int64), ("last_pkt", U32), ("done", U8)]


class RxQp(C.Structure):
    _fields_ = [("expected", U32), ("last_nack", U32), ("nack_timer", C.c_int64)]


class MmuPort(C.Structure):
    _fields_ = [("ing", U32), ("hdrm", U32), ("egr", U32), ("paused", U32)]


class MmuSwitch(C.Structure):
    _fields_ = [("shared_used", U32), ("total_hdrm", U32), ("total_rsrv", U32)]


_ull, _qr, _cp, _np, _qs = C.c_ulonglong, C.POINTER(QpRate), C.POINTER(CcParams), C.POINTER(NicParams), C.POINTER(QpSend)
_sw, _pt, _u32p = C.POINTER(MmuSwitch), C.POINTER(MmuPort), C.POINTER(C.c_uint)

# the rate rules: in both shims
SIG_CC = {
    "rc_failed": (C.c_int, []),
    "rc_sizes": (None, [C.POINTER(C.c_int)]),
    "rc_ns_seconds": (C.c_longlong, [C.c_double]),
    "rc_tx": (C.c_longlong, [_ull, C.c_uint, C.c_int]),
    "rc_node_ip": (C.c_uint, [C.c_int]),
    "rc_ecmp": (C.c_uint, [C.c_uint] * 4),
    "rc_hop_make": (_ull, [_ull, _ull, C.c_uint, _ull, C.c_uint]),
    "rc_hop_time_delta": (_ull, [_ull, _ull]),
    "rc_hop_bytes_delta": (_ull, [_ull, _ull, C.c_uint]),
    "rc_hop_u": (C.c_double, [_ull, _ull, C.c_uint, _ull, C.c_uint, C.POINTER(_ull)]),
    "rc_dcqcn": (C.c_uint, [_qr, _cp, C.c_int]),
    "rc_dctcp": (None, [_qr, _cp, C.c_uint, C.c_int]),
    "rc_hpcc": (C.c_int, [_qr, _cp, C.POINTER(_ull), C.c_int, C.c_int]),
    "rc_paced": (C.c_longlong, [C.c_longlong, C.c_int, _ull, _ull, C.c_uint]),
}
# the NIC, buffer and event-order rules: in the CPU shim
SIG_REST = {
    "rc_nic_sizes": (None, [C.POINTER(C.c_int)]),
    "rc_frame_sizes": (None, [_np, C.c_uint, C.POINTER(C.c_uint)]),
    "rc_next_qindex": (C.c_int, [_np, C.c_uint, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_longlong, _qr, _qs]),
    "rc_rx_check": (C.c_int, [_np, C.POINTER(RxQp), C.c_uint, C.c_uint, C.c_longlong]),
    "rc_ack_received": (C.c_uint, [_np, _cp, _qr, _qs, C.c_uint, C.c_int, C.c_int, C.POINTER(_ull), C.c_int]),
    "rc_qp_start": (None, [_np, _qr, _qs, _ull, _ull, C.c_uint, _ull, C.c_longlong]),
    "rc_next_data": (C.c_uint, [_np, _qr, _qs, C.c_longlong, C.c_int, C.POINTER(C.c_uint)]),
    "rc_next_send_at": (C.c_longlong, [_np, C.POINTER(C.c_int), C.c_int, C.c_longlong, _qr, _qs]),
    "rc_mmu_admit": (C.c_uint, [C.c_uint, _sw, _pt, C.c_uint, C.c_uint, _pt, C.c_uint, C.c_int]),
    "rc_mmu_release": (C.c_uint, [C.c_uint, _sw, _pt, C.c_uint, _pt, C.c_uint, C.c_int, C.c_uint, C.c_uint, C.c_double, C.c_int, C.c_double,
                                  C.POINTER(C.c_int)]),
    "rc_int_stamp": (None, [C.POINTER(_ull), C.POINTER(C.c_ushort), C.c_longlong, _ull, C.c_uint, _ull, C.c_uint]),
    "rc_ecmp_choice": (C.c_int, [C.c_int, C.c_int, C.c_uint, C.c_int, C.c_uint, C.c_int]),
    "rc_event_code": (C.c_uint, [C.c_longlong, C.c_int]),
    "rc_chain_hash": (_ull, [_ull, C.c_uint]),
    "rc_chain_order": (C.c_int, [_u32p, C.c_int, C.c_uint, _ull, _u32p, C.c_int, C.c_uint, _ull, _u32p]),
}


def build(out_dir, gpu=False):
    """The shim, built into out_dir and bound (gpu: the device shim, the rate rules only)."""
    if gpu:
        so = Path(out_dir) / "librc_gpu.so"
        cmd = ["nvcc", "-std=c++17", "-O2", "--fmad=false", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
               f"-I{CSRC}", "-o", str(so), str(SHIM_GPU)]
    else:
        so = Path(out_dir) / "librc.so"
        cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC", f"-I{CSRC}", "-o", str(so), str(SHIM)]
    subprocess.run(cmd, check=True)
    lib = C.CDLL(str(so))
    for name, (res, args) in {**SIG_CC, **({} if gpu else SIG_REST)}.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    sizes = (C.c_int * 3)()
    lib.rc_sizes(sizes)
    assert (sizes[0], sizes[1]) == (C.sizeof(QpRate), C.sizeof(CcParams))
    if not gpu:
        lib.rc_nic_sizes(sizes)
        assert list(sizes) == [C.sizeof(NicParams), C.sizeof(QpSend), C.sizeof(RxQp)]
    return lib


def load_kat():
    """{function: [case dict, ...]} of the reference's known answers."""
    raw = json.loads(gzip.decompress(KAT.read_bytes()))
    return {fn: [dict(zip(g["keys"], r)) for r in g["rows"]] for fn, g in raw.items()}


def dbl(h):
    """A double from the hex string of its bits."""
    return struct.unpack("<d", struct.pack("<Q", int(h, 16)))[0]


def bits(x):
    """The hex string of a double's bits."""
    return "0x%016x" % struct.unpack("<Q", struct.pack("<d", x))[0]


def params(row):
    """CcParams from a case's fields."""
    P = CcParams()
    for k in ("rpg_threshold", "rai", "rhai", "min_rate", "dctcp_rai", "mi_thresh", "sample_feedback", "int_multi", "mtu", "clamp"):
        setattr(P, k, row[k])
    for k in ("g", "rate_first_cnp", "u_target"):
        setattr(P, k, dbl(row[k]))
    return P


def sub(row, pre):
    """The fields of a case under a prefix ("a.": the state before an event, "b.": after)."""
    return {k[len(pre):]: v for k, v in row.items() if k.startswith(pre)}


def state(d):
    """A queue pair's rate state from a case's fields (before or after an event)."""
    q = QpRate()
    for k in ("rate", "max_rate", "target", "snd_nxt", "base_rtt", "win", "alpha_cnp", "dec_cnp", "first_cnp", "rp_stage", "cur_rate",
              "high_seq", "ecn_cnt", "batch", "ca_state"):
        if k in d:
            setattr(q, k, d[k])
    q.alpha = dbl(d["alpha"])
    if "u" in d:
        q.u = dbl(d["u"])
    q.last_update_seq, q.inc_stage = d["lus"], d["inc"]
    q.hop[:] = d["hop"]
    return q


def same(q, d):
    """Whether the fields of q that a case's state holds equal it (pacing is the caller's check)."""
    want = dict(d)
    got = {k: getattr(q, k) for k in want if hasattr(q, k) and k not in ("alpha", "u", "hop")}
    got.update(alpha=bits(q.alpha), lus=q.last_update_seq, inc=q.inc_stage, hop=list(q.hop))
    if "u" in want:
        got["u"] = bits(q.u)
    for k in ("next_avail", "last_pkt"):
        got[k] = want[k]
    return got == want
