// Model-specific code generation for the fused likelihood kernel.
//
// The reference evaluates resonance lineshapes through a bytecode interpreter
// or an NVRTC "materialise" pass that writes F and dF/dtheta for every event
// into an FP64 buffer (src/JITCustom.cu:654-711, 1148-1180). Here the whole
// per-event lineshape product of every amplitude column, with exact
// parameter derivatives (forward-mode jets), is emitted as straight-line CUDA
// C and compiled into the fused kernel, so nothing per-parameter is stored.
#pragma once

#include "model.hpp"

#include <string>
#include <vector>

namespace ctpwa {

// One per-event kinematic quantity cached at init (see angular.cuh AG_K_*).
struct KinSlot {
    int type;
    int group;
    int a, b, c;  // particle indices in the group
};

struct GeneratedModel {
    std::string header;          // model.cuh text
    std::string dual_header;     // model_dual.cuh text: the lineshapes in dual numbers (Hessian)
    std::vector<KinSlot> slots;  // kinematic cache layout
    int nplane = 0;              // angular planes = sum over groups of nSL
    int npol = 1;                // polarisation states per plane
    int ngrad = 0;               // gradient sums per thread: 2 nA + nTheta
    std::vector<int> group_plane0;
    int nder = 0;
    int nterm = 0;               // lineshape terms (one per amplitude column, more with identical particles)
    int nconst = 0;              // parameter-only subexpressions kept per call
    // per-event frontier tables (parameter-independent values the per-call
    // code reads): FP64 table rows; mixed form FP32 and FP64 rows
    int nev64 = 0;
    int nevf = 0;
    int nevd = 0;
};

GeneratedModel generateModel(const Model& m);

// Custom-expression syntax check (throws std::runtime_error like the reference parser).
void checkCustomExpr(const std::string& expr, const std::vector<std::string>& params);

}  // namespace ctpwa
