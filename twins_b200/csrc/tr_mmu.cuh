// twins-b200: the RDMA model's switch buffer rules (SwitchMmu of the HPCC fork of ns-3.17 that the
// reference's twins-rdma restates, for the data priority): ingress admission with a reserve, a
// shared pool under a dynamic threshold and per-port headroom, PFC PAUSE and RESUME, the release
// when a frame leaves, ECN marking at dequeue (RED between Kmin and Kmax) and the INT stamp of an
// HPCC data frame; and the ECMP choice of an egress port. Host and device functions; queues, links,
// the ECN random stream and event order are the caller's. Bit-exact with the reference's functions
// (src/rdma/rstep.cuh), which the oracle's known-answer vectors pin.
#pragma once
#include "tr_cc.cuh"

namespace tr
{

constexpr uint32_t MMU_RESERVE = 4 * 1024, MMU_RESUME_OFFSET = 3 * 1024;

// a port's buffer counters: as ingress (bytes held in its reserve and shared pool, in its headroom,
// whether it sent PAUSE) and as egress (bytes queued for it)
struct MmuPort
{
    uint32_t ing, hdrm, egr, paused;
};

// a switch's: its shared pool's use and the headroom and reserve it set aside for all ports
struct MmuSwitch
{
    uint32_t shared_used, total_hdrm, total_rsrv;
};

// the shared pool a port may still fill before PAUSE: what the buffer has left, shifted by the
// port's pfc_a_shift (reference: src/rdma/rstep.cuh:2196-2203)
TR_HD uint32_t pfc_threshold(uint32_t buffer_size, const MmuSwitch &sw, uint32_t shift)
{
    return (buffer_size - sw.total_hdrm - sw.total_rsrv - sw.shared_used) >> shift;
}
TR_HD uint32_t shared_part(const MmuPort &p) { return p.ing > MMU_RESERVE ? p.ing - MMU_RESERVE : 0; }

enum : unsigned
{
    MMU_DROP = 1,   // not admitted
    MMU_PAUSE = 2,  // the ingress port sends PAUSE
    MMU_MARK = 4,   // ECN: congestion experienced
    MMU_RESUME = 8  // the ingress port sends RESUME
};

// a data-priority frame of `size` bytes in on port `in` (headroom cap hdrm_cap, shift) for port
// `out` (CheckIngressAdmission, UpdateIngressAdmission, UpdateEgressAdmission, CheckAndSendPfc):
// dropped when it fits neither the headroom nor the threshold; else it fills the reserve, then the
// shared pool up to the threshold, then the headroom; PAUSE when headroom is in use or the shared
// part reaches the threshold (never on an NVSwitch) (reference: src/rdma/rstep.cuh:2411-2451)
TR_HD unsigned mmu_admit(uint32_t buffer_size, MmuSwitch &sw, MmuPort &in, uint32_t hdrm_cap, uint32_t shift, MmuPort &out, uint32_t size,
                         bool nvswitch)
{
    const uint32_t th = pfc_threshold(buffer_size, sw, shift);
    if (size + in.hdrm > hdrm_cap && size + shared_part(in) > th)
        return MMU_DROP;
    const uint32_t nb = in.ing + size;
    if (nb <= MMU_RESERVE)
        in.ing += size;
    else if (nb - MMU_RESERVE > th)
        in.hdrm += size;
    else
    {
        in.ing += size;
        sw.shared_used += size < nb - MMU_RESERVE ? size : nb - MMU_RESERVE;
    }
    out.egr += size;
    if (!nvswitch && !in.paused && (in.hdrm > 0 || shared_part(in) >= pfc_threshold(buffer_size, sw, shift)))
    {
        in.paused = 1;
        return MMU_PAUSE;
    }
    return 0;
}

// a data-priority frame of `size` bytes leaves port `out`, having come in on `in`
// (RemoveFromIngressAdmission, RemoveFromEgressAdmission, ShouldSendCN, CheckAndSendResume): the
// headroom gives back first, then the reserve and shared pool; with ECN the frame is marked when
// the egress queue is above kmax, or above kmin with probability pmax (egr - kmin) / (kmax - kmin)
// against draw() (a uniform number of the port's stream, drawn only there); a paused ingress
// resumes once its headroom is empty and its shared part is empty or RESUME_OFFSET below the
// threshold (reference: src/rdma/rstep.cuh:2318-2371)
template <class Draw>
TR_HD unsigned mmu_release(uint32_t buffer_size, MmuSwitch &sw, MmuPort &in, uint32_t in_shift, MmuPort &out, uint32_t size, bool ecn,
                           uint32_t kmin, uint32_t kmax, double pmax, bool nvswitch, Draw draw)
{
    unsigned res = 0;
    const uint32_t from_hdrm = in.hdrm < size ? in.hdrm : size;
    const uint32_t sh = shared_part(in);
    const uint32_t from_shared = size - from_hdrm < sh ? size - from_hdrm : sh;
    in.hdrm -= from_hdrm;
    in.ing -= size - from_hdrm;
    sw.shared_used -= from_shared;
    out.egr -= size;
    if (ecn && !nvswitch)
    {
        bool mark = false;
        if (out.egr > kmax)
            mark = true;
        else if (out.egr > kmin)
            mark = draw() < pmax * (double)(out.egr - kmin) / (double)(kmax - kmin);
        if (mark)
            res |= MMU_MARK;
    }
    if (in.paused && !nvswitch)
    {
        const uint32_t su = shared_part(in);
        if (in.hdrm == 0 && (su == 0 || su + MMU_RESUME_OFFSET <= pfc_threshold(buffer_size, sw, in_shift)))
        {
            in.paused = 0;
            res |= MMU_RESUME;
        }
    }
    return res;
}

// the INT stamp of an HPCC data frame leaving a port: hop word nhop % MAX_HOP takes (now, the
// port's bytes sent, its queue's bytes, its rate), and the count grows (reference:
// src/rdma/rstep.cuh:2372-2381)
TR_HD void int_stamp(uint64_t *hops, uint16_t &nhop, int64_t now, uint64_t tx_bytes, uint32_t queue_bytes, uint64_t bps, uint32_t multi)
{
    if (nhop == 0xFFFF)
        return;
    hops[nhop % MAX_HOP] = hop_make((uint64_t)now, tx_bytes, queue_bytes, bps, multi);
    nhop++;
}

// the egress port of a data frame (or its ACK, whose addresses and ports are swapped) among n
// equal-cost ports (SwitchNode::GetOutDev): the switch's ECMP hash of the source and destination
// addresses and ports (destination port 100), modulo n; src and dst are the data's hosts, numbered
// in the world (reference: src/rdma/rstep.cuh:2386-2409)
TR_HD int ecmp_choice(int src, int dst, uint32_t sport, bool data, uint32_t seed, int n)
{
    const int a = data ? src : dst, b = data ? dst : src;
    const uint32_t ports = data ? (sport | 100u << 16) : (100u | sport << 16);
    return (int)(ecmp_hash(node_ip(a), node_ip(b), ports, seed) % (uint32_t)n);
}

} // namespace tr
