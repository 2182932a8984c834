// twins-b200: the simulation state in device memory.
//
// Layout (all worlds of a batch side by side; ids are global unless marked world-local):
//   hosts       HostRec[H] + an egress ring of Frame[ring] each + active lists
//   switches    SwRec[S] (its world, first port, port count) ; ports PortRec[P] + rings
//   links       a host h sends on link h, port p on link H + p; per link and slot NB x MAX_TX frames
//   connections SndRec[C] (the sender's record) and RcvRec[C] (the receiver's), each touched by
//               one host only; per-connection rings for the sent list / RTT history and the
//               receiver's out-of-order blocks
//   messages    MsgRec[M]: the application's flows over connections
#pragma once
#include "tb_common.cuh"
#include "tb_host.h" // (the staging sizes SW_STAGE*)

namespace tb
{

// a world's topology and parameters (read-only on the device)
struct WorldDesc
{
    int kind;                 // TOPO_*
    int k, hk;                // ports per switch (FatTree k; leaf-spine max(hpl + spines, leaves))
    int leaves, spines, hpl;  // leaf-spine
    int ecmp_n;               // equal-cost uplinks a flow hash picks among (FatTree k/2, spines, 1)
    int H1, S1;               // hosts, switches
    int host0, sw0, conn0, msg0; // the world's first host, switch, connection, message
    int n_msgs;
    uint8_t cc, fin, spray, pad;
    int red_k, qcap;
    // topology files (TOPO_GRAPH), world-local ids; per epoch of link failures
    const int *host_sw;
    const uint8_t *host_port;
    const uint32_t *rt_off; // [epoch][S1][S1]
    const uint8_t *rt_n, *rt_ports;
    const uint8_t *port_dn; // [epoch][S1][k]
    const int64_t *fail_t;  // ps
    int n_fail;
};

// a connection's sent-list ring (and RTT history): an item per segment, message and FIN at most,
// capped at 65536, rounded up to a multiple of 8: the ring's flags are 32-bit words of eight
// positions (cap / 2 of the cap flag bytes the connection owns), and with every capacity a
// multiple of 8 every connection's offset, and so its words, are aligned
TB_HD uint32_t sent_list_cap(uint64_t segs)
{
    const uint64_t n = segs < 8 ? 8 : segs > 65536 ? 65536 : segs;
    return (uint32_t)((n + 7) & ~7ull);
}

// the sending side of a connection (TcpSocketBase, TcpTxBuffer, the congestion control)
struct SndRec
{
    // read-only
    int world, src_local, dst_local;
    uint32_t hash_data, hash_ack;
    int m_first, m_cnt; // messages (global ids, consecutive)
    uint32_t it_cap;    // sent-list / RTT-history ring capacity
    uint64_t it_off;
    // application and socket
    int m_due, m_wr, m_dn;
    uint8_t st, cong, fin, fin_on;
    uint32_t tail, una, nxt, high;
    uint32_t cwnd, ssthresh, dupacks;
    uint32_t it_head, it_n, h_head, h_n;
    uint32_t sack_b, lost_b, rtx_b, cand_b, sack_n, cand_lo, hisack; // the sent list's byte counters, sacked items, first-candidate bound, highest sack
    uint8_t sack_seen, recover_active, first_partial, cwnd_limited;
    uint32_t recover, cwnd_cnt, ack_rem;
    // TcpCubic
    uint32_t cub_cnt, cub_lastmax, cub_origin, cub_endseq, cub_samples, cub_ackcnt, cub_tcpcwnd;
    uint8_t cub_found, s_ce, ecn_s, next_seq_flag;
    double cub_k;
    int64_t cub_delaymin, cub_epoch, cub_roundstart, cub_lastack, cub_currrtt;
    // ECN / DCTCP
    int64_t ecn_echo_seq, ecn_cwr_seq;
    double alpha;
    uint32_t acked_total, acked_ecn, next_seq;
    uint8_t syn_tries, pad0[3];
    // RTT and timers
    int64_t srtt, rttvar, rto, rto_at, timing_time, syn_at;
    Chain rchain; // the retransmission (or SYN) timer's
    Chain schain; // the deferred SendPendingData's
};

// the receiving side (TcpRxBuffer, delayed ACKs, DCTCP's CE state, the closing states)
struct RcvRec
{
    int world, src_local, dst_local;
    uint32_t hash_ack;
    uint32_t oo_cap;
    uint64_t oo_off;
    uint32_t bytes;             // the connection's bytes (all its messages)
    uint8_t fin_on, up, est, st;
    int64_t fin_seq, synack_t, srtt, rttvar, last_at, frx_at, syn_at, delack_at, ecn_ce_seq;
    uint32_t rcv_nxt, ooo_n, ooo_h, prior_rcv_nxt;
    uint8_t last_n, syn_n, delack_count, ce_state, prior_flag, reserved, ecn_r, pad0;
    Chain dchain; // delayed ACK, SYN-ACK retransmission, LastAckTimeout
    Chain fchain; // the FIN+ACK's own retransmission
};

struct MsgRec
{
    int conn;
    uint32_t end;      // one past its last byte in the connection's stream
    int64_t start;     // ps
    int64_t est, done; // ps, -1: not yet
};

struct HostRec
{
    int world, local;
    int q_head, q_size;         // egress ring
    int64_t link_free, last_start;
    int n_snd, n_rcv;           // active connections as sender / receiver
    int pend_next, pend_end;    // the host's application events (indices into pend_msg)
    int64_t wake;               // earliest slot it must run without input
    int in_link;
    int pad;
    Chain last;                 // the chain of its transmission in progress
};

struct PortRec
{
    int q_head, q_size;
    int64_t link_free, last_start;
    int red_k, qcap;
    int in_link;                // the link arriving at this port (-1: unused)
    int pad;
    Chain last;
};

struct SwRec
{
    int world, local;
    int port0, k; // its first port, ports
};

// counters (one array per world is kept by the host; the device counts globally and per world)
enum : int
{
    EV_DROPS = 0,
    EV_MARKS,
    EV_RETX,
    EV_RTO,
    EV_TIES,      // undecided chain comparisons
    EV_HOST_PKT,  // packet-events at hosts (frame arrivals handled)
    EV_SW_PKT,    // packet-events at switch ports
    EV_OVF_ACT,   // capacity overflows: active lists, due timers, rings, out-of-order blocks, tx-cap
    EV_OVF_DUE,
    EV_OVF_RING,
    EV_OVF_OOO,
    EV_OVF_TX,
    EV_BARRIER_TIMEOUT,
    EV_HOST_SND,    // packet-events at hosts that reach a connection's sending side
    EV_HOST_FRAMES, // frames hosts emitted
    EV_N = 16
};

// the slot controller: barrier, time, idle skip, finish
struct SlotCtl
{
    unsigned arrive;
    unsigned gen;
    int64_t slot;
    unsigned act_cur, act_prev;
    unsigned long long next_wake;
    unsigned flows_done;
    int finished;
    int error;
    int pad;
    long long slots_run;
    // TB_PROFILE builds: per-slot maxima of a host unit's and a switch unit's time, summed over
    // slots, the slots' own time, and host / switch phase times (ns, the GPU's global timer)
    unsigned long long prof_host_max, prof_sw_max, prof_host_sum, prof_sw_sum, prof_slot_sum, prof_release;
    unsigned long long prof_phase[16];
};

// Per world: the slot rule of the reference's ticket block (src/kernel.cuh:79-112) applied to each
// world of a batch on its own, so that a world that is finished, or quiet until a timer, costs
// its entities nothing. Slots here are the launch's (global) slots; a world's own time starts at
// global slot `t0` (0 in a batch; the admission slot of a world that joins a running launch), and
// its entities run in world-local slots t - t0. `next` is the next global slot the world's
// entities run (INT64_MAX: all its messages are done); `act` / `prev` whether any of its entities
// sent or held frames in this and the previous slot; `wake` the earliest global wake-up its hosts
// reported in this slot.
// A batch launch without a grid-wide barrier (free_kernel) keeps each world on a barrier of its
// own: `run` is the slot its units run now (RUN_PARKED between launches), `arrive` how many of its
// `units` (in the launch's unit list) have done it, `budget` the slots it may still run in this
// launch, `last` the last slot it ran.
constexpr int64_t RUN_PARKED = -1;
struct WorldCtl
{
    int64_t next;
    unsigned long long wake;
    unsigned act, prev;
    unsigned fdone; // messages done
    unsigned pad;
    int64_t t0;
    int64_t run, last;
    unsigned arrive, units, budget, pad2;
};

// one enqueue at an egress queue, as the reference's --qtrace records it (src/model.h:313-320):
// the enqueue time (ps), the ns-3 node (hosts 0..H-1, then switches) and device (a host's NIC 1,
// switch port p + 1), the packet's source and destination host, its sequence (data) or ack
// number, length, the queue disc's length after the enqueue and the flags. Recorded by the trace
// build (TB_QTRACE) only.
struct QRec
{
    int64_t ts;
    int32_t node, dev, src, dst;
    uint32_t sa;
    uint16_t len, qlen;
    uint8_t flags, pad[3];
};

#if defined(TB_PROFILE) && defined(__CUDACC__)
__device__ __forceinline__ unsigned long long prof_now()
{
    unsigned long long t = 0;
#if defined(__CUDA_ARCH__)
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
#endif
    return t;
}
#define TB_PHASE_START unsigned long long prof_t0 = prof_now();
#define TB_PHASE(i)                                                   \
    {                                                                 \
        unsigned long long prof_t1 = prof_now();                      \
        atomicAdd(&s.ctl->prof_phase[i], prof_t1 - prof_t0);          \
        prof_t0 = prof_t1;                                            \
    }
#else
#define TB_PHASE_START
#define TB_PHASE(i)
#endif

struct Sim
{
    int W, H, S, P, L, C, M;
    int ring;           // egress ring capacity (max queue limit + 2)
    int act_cap;        // active-list capacity per host
    int64_t max_slots;
    const WorldDesc *worlds;
    HostRec *hosts;
    SwRec *sws;
    PortRec *ports;
    Frame *host_ring, *port_ring;
    int *act_snd, *act_rcv; // [H][act_cap]
    const int *pend_msg;
    SndRec *snd;
    RcvRec *rcv;
    MsgRec *msgs;
    uint32_t *it_start;
    uint8_t *it_fl;
    uint32_t *h_seq, *h_end;
    int64_t *h_t;
    uint32_t *oo_s, *oo_e;
    Frame *msg;          // [NB][L][MAX_TX]
    int64_t *msg_tag;    // [NB][L] slot << 16 | count (an old slot reads as empty)
    Rng *sw_rng;         // [S] (spraying worlds)
    uint8_t *sw_up;      // [S][kmax * 2 * MAX_TX] per-packet route choices (spraying)
    int64_t *sw_ts;      // [S][kmax * 2 * MAX_TX] egress sorting scratch
    uint32_t *sw_ref;
    int kmax;
    const double *cub_k_tab; // pow(n / 0.4, 1/3) from the host libm, n < cub_k_n
    int cub_k_n;
    unsigned long long *ev;  // [EV_N]
    unsigned long long *ev_w; // [W][EV_N]
    SlotCtl *ctl;
    WorldCtl *wctl;           // [W]
    // the units a launch runs (null: all): host units (host_lanes hosts each) of the worlds still
    // running, then host_units + switch; rebuilt between launches
    const int *unit_list;
    int n_list;
    // the free-running batch kernel: per list entry the last slot its unit ran (reset each launch),
    // per world its units in the list
    int64_t *unit_done;
    const unsigned *w_units;
    // the enqueue trace (trace build; null: off): records of enqueues with from <= time < until
    QRec *qtrace;
    unsigned long long *qtrace_cnt;
    unsigned long long qtrace_n;
    int64_t qtrace_from, qtrace_until;
};

} // namespace tb
