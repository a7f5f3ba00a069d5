// Model lowering: Config -> groups (chain x intermediate J^P), blocks
// (resonance combinations), amplitude columns, theta slots, coupling map,
// parameter names.
//
// Restates, for the likelihood path:
//   - Amp2BD::ComSL spin-orbit enumeration           src/AmpGen.cu:69-129
//   - AmpCasDecay chain bookkeeping / node masses    src/AmpGen.cu:405-480, 655-780
//   - DecayInfo amplitude names + coupling builder   src/Info.cu:43-357
//   - CouplingMatrixBuilder::buildWithTrans           src/Parameters.cu:586-735
//   - vspace remap of the coupling matrix             src/Analysis.cu:4382-4478
//   - polarisation map                                src/Analysis.cu:4249-4322
//   - calculateAmplitudes block/site order            src/Analysis.cu:4481-4830
//   - AmpCalc::addBlock theta slots, same-name and
//     trans sharing, default bounds                   src/AmpGen.cu:2009-2242
//   - AmpCalc::applyVarEqual                          src/AmpGen.cu:2244-2342
//   - Resonance model registry / param names          src/Resonance.cu:14-420
#pragma once

#include "config.hpp"

#include <map>
#include <string>
#include <utility>
#include <vector>

namespace ctpwa {

struct SLPair {
    int S;  // 2s+1
    int L;
};

enum class ModelType : int { BWR = 0, BW = 1, ONE = 2, Flatte = 3, Hist = 4, Custom = 5, GS = 6, Interp = 7 };
const char* modelTypeName(ModelType t);

// Daughter-mass source of a breakup momentum q0 = q(m0, md1, md2)
// (Q0MassDep, include/SymbolicDiff.cuh:130-134)
enum class MassSource : int { Fixed = 0, M0Param = 1, Event = 2 };

struct ModelNode {
    std::string mother_name, d1_name, d2_name;
    int mother = -1, d1 = -1, d2 = -1;  // indices in the group's particle table
    int dj = 1, dj1 = 1, dj2 = 1;       // 2J+1
    int par[3] = {1, 1, 1};
    double mass[3] = {-1, -1, -1};      // config masses; -1 for intermediates
    bool has_bf = true;
    double bf_d = 3.0;
    bool p_break = false;
    int l_min = 0;
    std::vector<SLPair> sls;
};

struct Group {
    std::string chain_name;
    std::vector<std::string> particle_names;  // alphabetical index space
    std::vector<int> particle_spin;           // 2J+1 per index
    std::vector<ModelNode> nodes;             // decay-step order
    std::vector<std::vector<int>> sl_combs;   // per combination: SL index per node
    // Contraction result: label order (particle indices) and tensor size.
    std::vector<int> final_labels;
    int tensor_size = 1;
    // Momentum reconstruction: for each particle index, its source.
    //   input_slot >= 0 : final-state particle read from the sample (Data.order slot)
    //   input_slot == -1: parent (sum of all finals)
    //   input_slot == -2: intermediate = sum of its two daughters (sum_a, sum_b)
    std::vector<int> input_slot;
    std::vector<std::pair<int, int>> sum_of;
    std::vector<int> build_order;  // particle indices in an order where sums are ready
    // Identical-particle symmetrisation (src/AmpGen.cu:194-405): a group whose
    // chain contains identical final-state particles has permutation
    // variants, each a copy of the group reading permuted final-state slots
    // (appended after all base groups). A block's amplitude is the signed sum
    // of its base group's and its variants' products.
    int base = -1;              // for a variant: index of its base group
    double sign = 1.0;          // for a variant: +1 (bosons) or sgn(permutation) (fermions)
    std::vector<int> variants;  // for a base group: indices of its variants
    int nSL() const { return (int)sl_combs.size(); }
};

struct ResInstance {
    std::string name;  // resonance name
    std::string tag;   // intermediate placeholder it sits on
    int J = 1, P = 1;
    ModelType type = ModelType::BWR;
    std::vector<double> params;            // ordered template values
    std::vector<std::string> param_names;  // ordered names (mass, width, g1, ...)
    std::vector<std::pair<double, double>> channels;
    std::map<std::string, std::string> options;
    int particle_idx = -1;  // in the group's particle table
    int node = -1;          // node whose mother is this resonance (-1: none)
    // theta source per parameter: global slot index or -1 (template value)
    std::vector<int> theta;
    // builtin-model AST settings (src/AmpGen.cu:2071-2101)
    int Lmin = 0;
    double d = 3.0;
    bool has_bf = true;
    MassSource md_src[2] = {MassSource::Event, MassSource::Event};
    double md_fixed[2] = {0.0, 0.0};
    std::vector<double> aux;  // Hist / Interp tables
};

struct Block {
    int group = -1;
    int site = 0;  // first amplitude column
    std::vector<ResInstance> res;
    bool free_path = false;  // re-evaluated per call (reference: nFree > 0)
};

struct ThetaSlot {
    int block, res, param;
    double init, lower, upper;
    std::string name;
};

struct CouplingMap {
    int n_free = 0;
    std::vector<int> amp_chain;     // amplitude -> free coupling index
    std::vector<double> ratio;      // amplitude -> real ratio (trans folding)
};

struct Model {
    Config cfg;
    std::vector<Particle> particles;
    std::string parent;                   // initial-state particle (not in Data.order)
    std::vector<std::string> final_order; // Data.order
    int npol = 1, npol_total = 1;
    std::vector<int> pol_map;             // output pol -> flattened tensor index (empty = identity)
    std::vector<Group> groups;
    std::vector<Block> blocks;
    std::vector<std::string> amplitude_names;
    std::vector<ThetaSlot> slots;
    CouplingMap coupling;
    std::vector<std::string> param_names;  // [coupling names..., theta slot names...]
    // gauss_constr: theta index -> (mu, sigma)
    std::vector<std::pair<int, std::pair<double, double>>> gauss;
    int fit_mode = 1;

    int nAmp() const { return (int)amplitude_names.size(); }
    int nVector() const { return coupling.n_free; }
    int nTheta() const { return (int)slots.size(); }
    int nParams() const { return 2 * nVector() + nTheta(); }
};

// Spin-orbit combinations of one two-body vertex (src/AmpGen.cu:69-129).
std::vector<SLPair> comSL(const int spins[3], const int parities[3], bool identical, bool boson,
                          int maxL, bool p_break, const std::vector<std::vector<int>>& sl_filter);

// Build the lowered model from a parsed config. Throws std::runtime_error.
Model buildModel(const Config& cfg, int fit_mode = 1);

// JSON description of the lowered model (test and tooling interchange).
std::string modelToJson(const Model& m);

}  // namespace ctpwa
