// TEST INFRASTRUCTURE — the oracle. Not product code: only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may build, call or run anything under oracle/.
//
// A plain, sequential CPU restatement of the reference TwiNS TCP model ("twins"): time advances
// in 1 us slots (the link propagation delay); in every slot each host, then each switch, handles
// its own events in timestamp order; simultaneous events are ordered by run-length-encoded
// ancestry chains. It follows, function by function, src/step.cuh (host TCP, egress FIFO with
// RED, switch forwarding), src/kernel.cuh:79-112 (slot barrier, exact idle skip) and
// src/main.cu:139-1015 (topologies, flows, connections, ECMP hashes). It always uses the
// reference's *general* forms (the TcpTxBuffer as a list of items, the TcpRxBuffer as sorted
// blocks, the RTT history as a list), which the reference validates against ns-3 on every run
// (validation/check_all.sh runs --general on lean-eligible workloads too).
//
// Containers are unbounded (no MAX_ACTIVE, MAX_DUE, ring or out-of-order caps); where the
// reference would overflow a capacity the oracle still computes ns-3's answer.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace oracle
{

enum Cc : uint8_t
{
    CC_NEWRENO = 0,
    CC_DCTCP = 1,
    CC_CUBIC = 2
};

enum TopoKind : int
{
    TOPO_FATTREE = 0,
    TOPO_LEAFSPINE = 1,
    TOPO_GRAPH = 2
};

struct LinkFail
{
    int64_t t_ns;
    int a, b; // switches (world-local)
    bool up;
};

struct Topology
{
    TopoKind kind = TOPO_FATTREE;
    int k = 4;                              // FatTree k
    int leaves = 16, spines = 8, hpl = 16;  // leaf-spine
    int g_hosts = 0, g_switches = 0;        // topology file
    std::vector<std::pair<int, int>> g_links; // endpoints: host h -> h, switch j -> -1 - j
    std::vector<LinkFail> fails;
};

struct FlowRow
{
    int src, dst;
    int64_t size, start_ns;
    int64_t conn = -1;
};

struct WorldSpec
{
    Topology topo;
    std::vector<FlowRow> flows;
    Cc cc = CC_DCTCP;
    int red_k = 30, qcap = 200;
    bool fin = false;
    bool spray = false;
    uint32_t rng_seed = 1;
    uint64_t rng_run = 1;
    int chain_runs = 9;            // 9: the reference's twins; 25: twins128
    int64_t max_slots = 2000000;
    bool have_hashes = false;      // per-flow ECMP hashes given (ns-3's), else computed
    std::vector<uint32_t> hash_data, hash_ack; // per message row (first row of each connection counts)
};

struct WorldResult
{
    std::vector<int64_t> est_ns, done_ns; // per message row, in file order (-1: not yet)
    std::vector<uint32_t> hash_data, hash_ack; // per message row (its connection's)
    uint64_t drops = 0, marks = 0, retx = 0, rtos = 0;
    uint64_t ties = 0;            // undecided chain comparisons (guessed orders)
    uint64_t events = 0;          // packet-events: frame arrivals handled at hosts and switch ports
    uint64_t host_events = 0, switch_events = 0;
    int64_t slots = 0;            // the slot reached (simulated time / 1 us)
    int64_t slots_run = 0;        // slots actually executed (idle slots skipped exactly)
    unsigned completed = 0;
};

std::vector<FlowRow> load_flows(const std::string &path, int hosts_per_world);
bool load_topofile(const std::string &path, Topology &t, std::string &err);
bool parse_fail_spec(const std::string &spec, Topology &t, std::string &err);
int hosts_of(const Topology &t);
WorldResult run_world(const WorldSpec &w);

} // namespace oracle
