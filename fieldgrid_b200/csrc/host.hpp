// Host-side model of one FDTD grid for the B200 engine: the product's counterpart of
// sims_field::fdtd::Sim (crates/sims-field/src/fdtd/sim.rs:173-189).
//
// Layout decision: the reference keeps ca/cb as six nn-long f32 arrays (24 B per node) and its
// GPU path re-indexes them into deduplicated (ca, cb) pairs with a u16 per edge (6 B per node,
// run.rs:61-100). This engine goes one step further: a node's three E edges form one triple
// {ca[3], cb[3]}, the triples are deduplicated into a class table, and each node stores one
// class id (1 B when there are at most 256 triples, 2 B up to 65536, else 4 B). Bulk material
// regions share a handful of triples, so the id array is the only per-node coefficient traffic.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace fg {

constexpr double C0 = 299792458.0;
constexpr double EPS0 = 8.8541878128e-12;
constexpr double MU0 = 1.25663706212e-6;
constexpr double ETA0 = 376.730313668;
constexpr double PI = 3.14159265358979323846;

struct Error {
    int code;
    std::string msg;
};

// One node of an axis: the 10 values run.rs:226-242 packs per node, slots as ints.
struct AxisNode {
    float inv_d, inv_dd, raw_inv_d, raw_inv_dd, be, ce, bh, ch;
    int32_t slot_e, slot_h;
};

// The same factors in f64 (before their rounding to f32), for the FP64 forward.
struct AxisNode64 {
    double inv_d, inv_dd, raw_inv_d, raw_inv_dd, be, ce, bh, ch;
    int32_t slot_e, slot_h;
};

struct Axis {
    size_t n = 0;
    std::vector<double> d, dd;
    std::vector<AxisNode> node;
    std::vector<AxisNode64> node64;
};

struct Edge {
    uint32_t comp;
    size_t at[3];
};

struct PortDef {
    std::vector<std::vector<Edge>> columns;
    double r = 0;
    bool reference_above = false;
};

struct SrcEdge {
    uint32_t comp;
    uint64_t id;
    float src;
};

struct Inductor {
    uint32_t comp;
    uint64_t id;
    float ke, ki;
};

struct SheetEdge {
    uint32_t comp;
    uint64_t id;
    double r;
    bool adaptive;
    uint64_t faces[2];
    double len, c;
};

struct DebyeEdge {
    uint32_t comp;
    uint64_t id;
    double dd;
};

struct WireH {
    uint64_t h;               // comp*nn + id of the H component
    uint64_t e[4];            // comp*nn + id of each E term
    float c[4];
};

struct Coef {                 // one node's three E edges
    float ca[3], cb[3];
};

struct HostSim {
    std::vector<double> line[3];
    size_t pml = 0;
    size_t n[3] = {0, 0, 0};
    size_t nn = 0;
    double dt = 0;
    Axis ax[3];
    std::vector<uint32_t> node_class;     // nn entries, or empty when node_class16 holds them
    std::vector<uint16_t> node_class16;   // nn entries when there are at most 65,536 classes
    uint32_t cls(size_t id) const { return node_class16.empty() ? node_class[id] : uint32_t(node_class16[id]); }
    std::vector<Coef> classes;
    std::vector<PortDef> ports;
    std::vector<std::vector<SrcEdge>> port_src;
    std::vector<Inductor> inductors;
    std::vector<SheetEdge> sheets;
    std::vector<float> sheet_table;
    size_t sheet_states = 0;
    std::vector<std::pair<double, double>> poles;
    std::vector<DebyeEdge> debye_edges;
    std::vector<WireH> wires;
    std::vector<float> cell_eps, cell_sig;   // per cell as given (empty: the defaults 1 and 0)

    size_t cells() const { return (n[0] - 1) * (n[1] - 1) * (n[2] - 1); }
    size_t idx(size_t i, size_t j, size_t k) const { return (i * n[1] + j) * n[2] + k; }
    float ca(uint32_t c, size_t id) const { return classes[cls(id)].ca[c]; }
    float cb(uint32_t c, size_t id) const { return classes[cls(id)].cb[c]; }
};

double time_step(const std::vector<double>* line);
void pulse_shape(double fc, double& t0, double& tau);

}  // namespace fg
