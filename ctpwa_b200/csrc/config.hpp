// config.yml schema -> in-memory configuration.
//
// Restates the reference's ConfigParser (src/Config.cu:138-1310,
// include/Config.cuh:11-190) for the parts that feed the likelihood path:
// Particles, Data, DecayChains (compact and expanded forms), Resonances
// (inline or external file), Constraints (maxL, bf_d, has_bf, fix_var,
// free_var, var_range, var_equal, gauss_constr, identical, trans, chains),
// precision, and the three-level barrier-factor scope resolution.
// The Plot section is accepted and ignored (plots are not part of this path).
#pragma once

#include <cmath>
#include <complex>
#include <map>
#include <set>
#include <string>
#include <utility>
#include <vector>

namespace ctpwa {

struct Particle {
    std::string name;
    int spin = 1;    // 2J+1
    int parity = 1;
    double mass = -1.0;
    std::string identical_group;
    std::vector<int> polarization_2m;  // allowed 2m values; empty = all states
    bool is_fermion() const { return (spin - 1) % 2 != 0; }
    bool is_polarized() const { return !polarization_2m.empty(); }
};

struct ResonanceConfig {
    std::string name;
    int J = -1;  // 2J+1; -1 = not given
    int P = 0;
    std::string type;
    std::vector<double> parameters;
    std::vector<std::vector<double>> channels;
    std::vector<int> free;  // {-1} = all, empty = none
    std::vector<std::vector<double>> free_range;
    std::map<std::string, std::string> options;
    bool has_bf = true;
    bool has_bf_explicit = false;
    double bf_d = NAN;
};

struct SpinChainConfig {
    std::vector<int> spin_parity;  // {2J+1, P}
    std::vector<std::string> resonances;
};

struct ResonanceChainConfig {
    std::string intermediate;
    std::vector<SpinChainConfig> spin_chains;
};

struct DecayStep {
    std::string mother;
    std::vector<std::string> daughters;
    bool has_bf = true;
    bool has_bf_explicit = false;
    double bf_d = NAN;
    bool p_break = false;
    std::vector<std::vector<int>> sl_filter;  // [2S+1, L]
};

struct DecayChainConfig {
    std::string name;
    std::vector<DecayStep> decay_steps;
    std::vector<ResonanceChainConfig> resonance_chains;
};

struct ConstraintConfig {
    std::vector<std::string> names;
    std::vector<std::complex<double>> values;
    std::string type;
};

struct Config {
    std::string config_file;
    std::vector<Particle> particles;
    std::vector<DecayChainConfig> decay_chains;
    std::map<std::string, ResonanceConfig> resonances;
    std::map<std::string, std::vector<std::string>> data_files;
    std::vector<std::string> data_order;
    std::vector<ConstraintConfig> constraints;
    int global_maxL = -1;
    double global_bf_d = 3.0;
    bool global_has_bf = true;
    std::string precision = "auto";
    std::map<std::string, double> fix_var;
    std::set<std::string> free_var;
    std::map<std::string, std::pair<double, double>> var_range;
    std::vector<std::vector<std::string>> var_equal;
    std::map<std::string, double> gauss_constr;
    std::vector<std::string> chain_filter;
    std::vector<std::string> warnings;

    // The reference treats a config without particles as invalid
    // (ConfigParser::isValid, include/Config.cuh:113).
    bool valid() const { return !particles.empty(); }
    const Particle* findParticle(const std::string& n) const;
};

// Parse a config file. Syntax errors in the file make the result invalid
// (the reference prints a warning and leaves the parser empty,
// src/Config.cu:243-246); semantic errors throw std::runtime_error.
Config loadConfig(const std::string& path);
Config loadConfigText(const std::string& text, const std::string& path_for_relative);

// "1", "1/2", "0.5" -> float (src/Config.cu:117-136)
float transJValue(const std::string& s);

}  // namespace ctpwa
