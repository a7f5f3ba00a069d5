// Event samples: four-momenta of the final-state particles and optional
// per-event weights.
//
// Restates readMomentaFromDat (src/Analysis.cu:58-176, "dat" branch) and
// readWeightsFromFile (src/Analysis.cu:292-400): a dat file holds one line
// "E px py pz" per final-state particle, particles in Data.order, events
// consecutive; the initial state is the sum of the final states. A weight
// spec is either a constant ([w]) or [dat, file] with one weight per line.
// Additionally an "npy" type reads a float64 array of shape (N, n_final, 4)
// (same content, binary) for large synthetic samples.
#pragma once

#include <string>
#include <vector>

namespace ctpwa {

struct Sample {
    long n = 0;
    int n_final = 0;
    std::vector<double> p4;       // [n][n_final][4]  (E, px, py, pz)
    std::vector<double> weights;  // empty = unit weights
};

// fileinfo = {type, path}; type "dat" or "npy". ROOT files are not supported.
Sample readSample(const std::vector<std::string>& fileinfo, int n_final);
// Weights for an existing sample: {"0.8"} (constant) or {"dat", path}.
std::vector<double> readWeights(const std::vector<std::string>& fileinfo, long n_events);

// Keep shard `rank` of `world` contiguous event blocks of a sample (and of
// its per-event weights, when given): events [n*rank/world, n*(rank+1)/world).
// Event-sharded evaluation over several devices (src/Analysis.cu:4210-4238
// splits its samples the same way).
void shardSample(Sample& s, std::vector<double>& weights, int rank, int world);

}  // namespace ctpwa
