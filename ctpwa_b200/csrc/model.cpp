// Model lowering (see model.hpp for the reference mapping).
#include "model.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <set>
#include <sstream>
#include <stdexcept>

namespace ctpwa {

const char* modelTypeName(ModelType t)
{
    switch (t) {
    case ModelType::BWR: return "BWR";
    case ModelType::BW: return "BW";
    case ModelType::ONE: return "ONE";
    case ModelType::Flatte: return "Flatte";
    case ModelType::Hist: return "Hist";
    case ModelType::Custom: return "Custom";
    case ModelType::GS: return "GS";
    case ModelType::Interp: return "Interp";
    }
    return "?";
}

std::vector<SLPair> comSL(const int spins[3], const int parities[3], bool identical, bool boson,
                          int maxL, bool p_break, const std::vector<std::vector<int>>& sl_filter)
{
    std::set<std::pair<int, int>> filt;
    for (const auto& f : sl_filter)
        if (f.size() >= 2) filt.insert({f[0], f[1]});
    std::vector<SLPair> out;
    const int tj1 = spins[0] - 1, tj2 = spins[1] - 1, tj3 = spins[2] - 1;  // 2J
    for (int tS = std::abs(tj2 - tj3); tS <= tj2 + tj3; tS += 2) {
        for (int tL = std::abs(tj1 - tS); tL <= tj1 + tS; tL += 2) {
            int L = tL / 2;
            int sign = (L % 2 == 0) ? 1 : -1;
            if (!(p_break || parities[0] == parities[1] * parities[2] * sign)) continue;
            if (identical) {
                int S = tS / 2;
                int pls = ((L + S) % 2 == 0) ? 1 : -1;
                if (pls != (boson ? 1 : -1)) continue;
            }
            if (maxL > 0 && L > maxL) continue;
            if (!filt.empty() && !filt.count({tS + 1, L})) continue;
            out.push_back({tS + 1, L});
        }
    }
    return out;
}

namespace {

ModelType parseModelType(const std::string& s)
{
    static const std::vector<std::pair<std::string, ModelType>> tab = {
        {"BWR", ModelType::BWR}, {"BW", ModelType::BW},         {"ONE", ModelType::ONE},
        {"Flatte", ModelType::Flatte}, {"GS", ModelType::GS},   {"Interp", ModelType::Interp},
        {"Hist", ModelType::Hist}, {"Custom", ModelType::Custom}};
    for (const auto& t : tab)
        if (t.first == s) return t.second;
    std::string lo = s;
    std::transform(lo.begin(), lo.end(), lo.begin(), ::tolower);
    for (const auto& t : tab) {
        std::string k = t.first;
        std::transform(k.begin(), k.end(), k.begin(), ::tolower);
        if (k == lo) return t.second;
    }
    throw std::runtime_error("Unknown model type: " + s);
}

std::vector<std::string> splitParamNames(const std::string& s)
{
    std::vector<std::string> out;
    size_t pos = 0;
    while (pos <= s.size()) {
        size_t c = s.find(',', pos);
        std::string n = (c == std::string::npos) ? s.substr(pos) : s.substr(pos, c - pos);
        size_t b = n.find_first_not_of(" \t");
        size_t e = n.find_last_not_of(" \t");
        if (b != std::string::npos) out.push_back(n.substr(b, e - b + 1));
        if (c == std::string::npos) break;
        pos = c + 1;
    }
    return out;
}

// Ordered parameter names/values of a resonance model (src/Resonance.cu:14-420).
void setParamsFromModel(ResInstance& r, const std::vector<double>& params)
{
    struct Spec {
        const char* name;
        bool optional;
    };
    std::vector<std::pair<std::string, bool>> specs;
    std::string prefix;
    switch (r.type) {
    case ModelType::BWR: specs = {{"mass", false}, {"width", false}, {"r", true}}; break;
    case ModelType::BW: specs = {{"mass", false}, {"width", false}}; break;
    case ModelType::ONE: specs = {{"mass", false}}; break;
    case ModelType::Flatte: specs = {{"mass", false}}; prefix = "g"; break;
    case ModelType::GS: specs = {{"mass", false}, {"width", false}}; break;
    case ModelType::Interp: break;
    case ModelType::Hist: specs = {{"mass", true}}; break;
    case ModelType::Custom: {
        auto it = r.options.find("params");
        if (it != r.options.end())
            for (const auto& n : splitParamNames(it->second)) specs.push_back({n, false});
        break;
    }
    }
    size_t required = 0;
    for (const auto& s : specs)
        if (!s.second) ++required;
    if (params.size() < required)
        throw std::runtime_error("Model '" + std::string(modelTypeName(r.type)) + "' requires at least " +
                                 std::to_string(required) + " parameter(s), got " + std::to_string(params.size()));
    r.params.clear();
    r.param_names.clear();
    for (size_t i = 0; i < specs.size() && i < params.size(); ++i) {
        r.param_names.push_back(specs[i].first);
        r.params.push_back(params[i]);
    }
    if (!prefix.empty())
        for (size_t i = specs.size(); i < params.size(); ++i) {
            r.param_names.push_back(prefix + std::to_string(i));
            r.params.push_back(params[i]);
        }
}

// Hist shape table (src/Resonance.cu:121-180)
std::vector<double> buildHistAux(const std::map<std::string, std::string>& o)
{
    auto get = [&](const char* k) {
        auto it = o.find(k);
        return it == o.end() ? std::string() : it->second;
    };
    std::string file = get("file"), bins = get("bins"), range = get("range");
    if (file.empty() || bins.empty() || range.empty())
        throw std::runtime_error("Hist model requires file, bins and range options");
    int nb = std::stoi(bins);
    if (nb < 2) throw std::runtime_error("Hist model needs bins >= 2");
    std::vector<double> rg;
    {
        std::stringstream ss(range);
        std::string tok;
        while (std::getline(ss, tok, ',')) rg.push_back(std::stod(tok));
    }
    if (rg.size() != 2 || rg[1] <= rg[0]) throw std::runtime_error("Hist model needs range lo,hi with hi > lo");
    std::ifstream f(file);
    if (!f.is_open()) throw std::runtime_error("Hist model: cannot open file " + file);
    std::vector<double> vals;
    double v;
    while (f >> v) vals.push_back(v);
    if ((int)vals.size() != nb)
        throw std::runtime_error("Hist model: file " + file + " has " + std::to_string(vals.size()) +
                                 " values, expected " + std::to_string(nb));
    std::vector<double> aux = {rg[0], rg[1], (double)nb};
    aux.insert(aux.end(), vals.begin(), vals.end());
    return aux;
}

// Interp table (src/Resonance.cu:75-119); file of "x re im" rows.
std::vector<double> buildInterpAux(const std::map<std::string, std::string>& o)
{
    int method = 1;
    auto it = o.find("method");
    if (it != o.end()) {
        if (it->second == "hist") method = 0;
        else if (it->second == "spline") method = 2;
    }
    it = o.find("file");
    if (it == o.end()) return {};
    std::ifstream f(it->second);
    if (!f) return {};
    std::vector<double> x, re, im;
    double a, b, c;
    while (f >> a >> b >> c) {
        x.push_back(a);
        re.push_back(b);
        im.push_back(c);
    }
    if (x.size() < 2) return {};
    double dx = x[1] - x[0];
    bool uniform = true;
    for (size_t i = 1; i < x.size(); ++i)
        if (std::fabs(x[i] - x[i - 1] - dx) > 1e-10) {
            uniform = false;
            break;
        }
    std::vector<double> aux;
    if (uniform) {
        aux = {(double)method, (double)x.size(), x[0], dx};
    } else {
        aux = {(double)-(method + 1), (double)x.size()};
        aux.insert(aux.end(), x.begin(), x.end());
    }
    aux.insert(aux.end(), re.begin(), re.end());
    aux.insert(aux.end(), im.begin(), im.end());
    return aux;
}

struct JPParticle {
    std::string name;
    int spin, parity;
};

struct AmpMapEntry {
    int amp_idx;
    std::string chain_key;
};

}  // namespace

namespace {

// Permutation variants of groups with identical final-state particles,
// following AmpCasDecay::buildPermTopologies (src/AmpGen.cu:194-405): the
// amplitude is summed over the full permutation group of each identical
// group's members present in the chain (the stabiliser swaps of two
// identical daughters of one decay step included), with sgn(permutation) for
// fermions and +1 for bosons. Several identical groups in one chain combine
// as the reference does: the non-identity elements of the groups are
// multiplied out pairwise (src/AmpGen.cu:366-385). Members that are
// intermediate resonances (whole subtrees permuted) are not supported.
void addIdenticalVariants(const Config& cfg, Model& m)
{
    const int nbase = (int)m.groups.size();
    for (int gi = 0; gi < nbase; ++gi) {
        const Group& G = m.groups[gi];
        std::map<std::string, std::vector<int>> members;  // identical group -> particle indices
        std::map<std::string, bool> boson;
        for (size_t i = 0; i < G.particle_names.size(); ++i) {
            const Particle* p = cfg.findParticle(G.particle_names[i]);
            if (!p || p->identical_group.empty() || G.input_slot[i] == -1) continue;
            members[p->identical_group].push_back((int)i);
            boson[p->identical_group] = !p->is_fermion();
        }
        std::vector<std::vector<int>> maps;  // non-identity variants: input_slot arrays
        std::vector<double> signs;
        bool first = true;
        for (const auto& kv : members) {
            const std::vector<int>& mem = kv.second;
            if (mem.size() < 2) continue;
            for (int i : mem)
                if (G.input_slot[i] < 0)
                    throw std::runtime_error("chain " + G.chain_name + ": identical particle " + G.particle_names[i] +
                                             " is not a final-state particle (subtree permutations are not supported)");
            const int n = (int)mem.size();
            std::vector<int> perm(n);
            for (int i = 0; i < n; ++i) perm[i] = i;
            std::vector<std::vector<int>> gmaps;
            std::vector<double> gsigns;
            while (std::next_permutation(perm.begin(), perm.end())) {
                // member i reads the momentum of member perm[i]
                std::vector<int> slots(G.input_slot.size(), 0);
                int inv = 0;
                for (int i = 0; i < n; ++i)
                    for (int j = i + 1; j < n; ++j)
                        if (perm[i] > perm[j]) ++inv;
                gmaps.push_back({});
                for (int i = 0; i < n; ++i) gmaps.back().push_back(perm[i]);
                gsigns.push_back(boson[kv.first] ? 1.0 : ((inv % 2) ? -1.0 : 1.0));
            }
            // as slot arrays over this identical group only (identity elsewhere)
            std::vector<std::vector<int>> gslots;
            for (const auto& pm : gmaps) {
                std::vector<int> sl = G.input_slot;
                for (int i = 0; i < n; ++i) sl[mem[i]] = G.input_slot[mem[pm[i]]];
                gslots.push_back(sl);
            }
            if (first) {
                maps = gslots;
                signs = gsigns;
                first = false;
            } else {
                std::vector<std::vector<int>> nm;
                std::vector<double> ns;
                for (size_t a = 0; a < maps.size(); ++a)
                    for (size_t b = 0; b < gslots.size(); ++b) {
                        std::vector<int> merged = gslots[b];
                        for (const auto& kv2 : members)
                            if (kv2.first != kv.first && kv2.second.size() >= 2)
                                for (int i : kv2.second) merged[i] = maps[a][i];
                        nm.push_back(merged);
                        ns.push_back(signs[a] * gsigns[b]);
                    }
                maps = std::move(nm);
                signs = std::move(ns);
            }
        }
        for (size_t v = 0; v < maps.size(); ++v) {
            Group var = m.groups[gi];
            var.variants.clear();
            var.input_slot = maps[v];
            var.base = gi;
            var.sign = signs[v];
            m.groups.push_back(var);
            m.groups[gi].variants.push_back((int)m.groups.size() - 1);
        }
    }
}

}  // namespace

Model buildModel(const Config& cfg, int fit_mode)
{
    if (!cfg.valid()) throw std::runtime_error("analysis not initialized: invalid or missing config file");
    if (fit_mode != 1)
        throw std::runtime_error("fit mode 0 (chain x step couplings) is not supported; use the default vspace mode (1)");
    Model m;
    m.cfg = cfg;
    m.fit_mode = fit_mode;
    m.particles = cfg.particles;
    m.final_order = cfg.data_order;

    // ---- polarisation (src/Analysis.cu:4249-4322) ----
    {
        int n = (int)m.particles.size();
        std::vector<int> dims(n), eff(n), os(n), ms(n);
        std::vector<std::vector<int>> keep(n);
        bool masked = false;
        for (int i = 0; i < n; ++i) {
            dims[i] = m.particles[i].spin;
            if (m.particles[i].is_polarized()) {
                masked = true;
                for (int tm : m.particles[i].polarization_2m) keep[i].push_back((dims[i] - 1 - tm) / 2);
            }
        }
        os[n - 1] = 1;
        for (int i = n - 2; i >= 0; --i) os[i] = os[i + 1] * dims[i + 1];
        m.npol_total = 1;
        for (int d : dims) m.npol_total *= d;
        for (int i = 0; i < n; ++i) eff[i] = keep[i].empty() ? dims[i] : (int)keep[i].size();
        ms[n - 1] = 1;
        for (int i = n - 2; i >= 0; --i) ms[i] = ms[i + 1] * eff[i + 1];
        m.npol = 1;
        for (int d : eff) m.npol *= d;
        if (masked) {
            m.pol_map.resize(m.npol);
            for (int out = 0; out < m.npol; ++out) {
                int rem = out, t = 0;
                for (int p = 0; p < n; ++p) {
                    int j = rem / ms[p];
                    rem %= ms[p];
                    int i = keep[p].empty() ? j : keep[p][j];
                    t += i * os[p];
                }
                m.pol_map[out] = t;
            }
        }
    }

    // ---- parent = the one config particle not in Data.order (src/Analysis.cu:85-103) ----
    {
        std::set<std::string> order(cfg.data_order.begin(), cfg.data_order.end());
        int n_missing = 0;
        for (const auto& p : m.particles)
            if (!order.count(p.name)) {
                m.parent = p.name;
                ++n_missing;
            }
        if (n_missing != 1)
            throw std::runtime_error("Particles must be the initial state plus the final states listed in Data.order");
        for (const auto& n : cfg.data_order)
            if (!cfg.findParticle(n)) throw std::runtime_error("Data.order lists unknown particle " + n);
    }

    // ---- trans chain links (src/Analysis.cu:4505-4523) ----
    std::map<std::string, std::set<std::string>> chain_linked;
    for (const auto& c : cfg.constraints) {
        if (c.type != "trans" || c.names.size() < 2) continue;
        std::vector<std::string> matched;
        for (const auto& cn : c.names)
            for (const auto& ch : cfg.decay_chains)
                if (ch.name.find(cn) != std::string::npos) {
                    matched.push_back(ch.name);
                    break;
                }
        for (size_t i = 0; i < matched.size(); ++i)
            for (size_t j = 0; j < matched.size(); ++j)
                if (i != j) chain_linked[matched[i]].insert(matched[j]);
    }
    std::map<std::string, std::vector<std::vector<std::string>>> chain_resonances;
    std::map<std::string, int> chain_comb_index;
    std::map<std::string, std::pair<int, int>> resonance_owners;
    std::map<std::pair<int, int>, std::pair<int, int>> conj_broadcast;
    std::vector<AmpMapEntry> amp_map;

    int gls = 0;
    for (const auto& chain : cfg.decay_chains) {
        // -- intermediate -> [J^P -> resonance list] (src/Info.cu:57-103) --
        std::map<std::pair<std::string, std::pair<int, int>>, std::vector<ResInstance>> irmap;
        std::vector<std::vector<JPParticle>> ips;
        for (const auto& rc : chain.resonance_chains) {
            std::vector<JPParticle> pj;
            for (const auto& sc : rc.spin_chains) {
                if (sc.spin_parity.size() < 2)
                    throw std::runtime_error("intermediate " + rc.intermediate + " needs [J: .., P: ..]");
                JPParticle ip{rc.intermediate, sc.spin_parity[0], sc.spin_parity[1]};
                std::vector<ResInstance> rl;
                for (const auto& rn : sc.resonances) {
                    auto it = cfg.resonances.find(rn);
                    if (it == cfg.resonances.end()) continue;
                    if (!(it->second.J < 0 || it->second.J == sc.spin_parity[0])) continue;
                    ResInstance r;
                    r.name = rn;
                    r.tag = rc.intermediate;
                    r.J = ip.spin;
                    r.P = ip.parity;
                    r.type = parseModelType(it->second.type);
                    r.options = it->second.options;
                    for (const auto& ch : it->second.channels)
                        if (ch.size() >= 2) r.channels.emplace_back(ch[0], ch[1]);
                    for (const auto& st : chain.decay_steps)
                        if (st.mother == rc.intermediate) {
                            r.options["d"] = std::to_string(st.bf_d);
                            r.options["has_bf"] = st.has_bf ? "1" : "0";
                            break;
                        }
                    setParamsFromModel(r, it->second.parameters);
                    if (r.type == ModelType::Hist) r.aux = buildHistAux(r.options);
                    if (r.type == ModelType::Interp) r.aux = buildInterpAux(r.options);
                    if (r.type == ModelType::Custom) {
                        if (!r.options.count("expr")) throw std::runtime_error("Custom model requires expr option");
                        if (r.param_names.size() > 16)
                            throw std::runtime_error("Custom model supports at most 16 free params");
                    }
                    rl.push_back(r);
                }
                irmap[{rc.intermediate, {ip.spin, ip.parity}}] = rl;
                pj.push_back(ip);
            }
            ips.push_back(pj);
        }
        std::vector<std::vector<JPParticle>> combs = {{}};
        for (const auto& pl : ips) {
            std::vector<std::vector<JPParticle>> t;
            for (const auto& c : combs)
                for (const auto& p : pl) {
                    auto nc = c;
                    nc.push_back(p);
                    t.push_back(nc);
                }
            combs = std::move(t);
        }


        for (const auto& comb : combs) {
            Group g;
            g.chain_name = chain.name;
            // -- nodes (src/Analysis.cu:4581-4663) --
            std::map<std::string, std::pair<int, double>> spinmass;  // name -> (spin, mass)
            for (const auto& p : m.particles) spinmass[p.name] = {p.spin, p.mass};
            for (const auto& st : chain.decay_steps) {
                if (st.daughters.size() != 2)
                    throw std::runtime_error("chain " + chain.name + ": every decay step needs two daughters");
                int spins[3] = {0, 0, 0}, pars[3] = {0, 0, 0};
                const std::string* names[3] = {&st.mother, &st.daughters[0], &st.daughters[1]};
                for (const auto& p : m.particles)
                    for (int k = 0; k < 3; ++k)
                        if (p.name == *names[k]) {
                            spins[k] = p.spin;
                            pars[k] = p.parity;
                        }
                for (const auto& jp : comb)
                    for (int k = 0; k < 3; ++k)
                        if (jp.name == *names[k]) {
                            spins[k] = jp.spin;
                            pars[k] = jp.parity;
                        }
                bool ident = false, boson = true;
                const Particle* p1 = cfg.findParticle(st.daughters[0]);
                const Particle* p2 = cfg.findParticle(st.daughters[1]);
                if (p1 && p2 && !p1->identical_group.empty() && p1->identical_group == p2->identical_group) {
                    ident = true;
                    boson = !p1->is_fermion();
                }
                ModelNode nd;
                nd.mother_name = st.mother;
                nd.d1_name = st.daughters[0];
                nd.d2_name = st.daughters[1];
                nd.dj = spins[0];
                nd.dj1 = spins[1];
                nd.dj2 = spins[2];
                for (int k = 0; k < 3; ++k) nd.par[k] = pars[k];
                nd.has_bf = st.has_bf;
                nd.bf_d = st.bf_d;
                nd.p_break = st.p_break;
                nd.sls = comSL(spins, pars, ident, boson, cfg.global_maxL, st.p_break, st.sl_filter);
                int lmin = -1;
                for (const auto& sl : nd.sls)
                    if (lmin < 0 || sl.L < lmin) lmin = sl.L;
                nd.l_min = lmin < 0 ? 0 : lmin;
                for (int k = 0; k < 3; ++k) {
                    auto it = spinmass.find(*names[k]);
                    nd.mass[k] = (it != spinmass.end()) ? it->second.second : -1.0;
                }
                g.nodes.push_back(nd);
            }
            // particle index space: sorted names (src/AmpGen.cu:663-680)
            {
                std::set<std::string> all;
                for (const auto& nd : g.nodes) {
                    all.insert(nd.mother_name);
                    all.insert(nd.d1_name);
                    all.insert(nd.d2_name);
                }
                for (const auto& p : m.particles) all.insert(p.name);
                g.particle_names.assign(all.begin(), all.end());
                auto idx = [&](const std::string& n) {
                    return (int)(std::lower_bound(g.particle_names.begin(), g.particle_names.end(), n) -
                                 g.particle_names.begin());
                };
                g.particle_spin.assign(g.particle_names.size(), 1);
                for (auto& nd : g.nodes) {
                    nd.mother = idx(nd.mother_name);
                    nd.d1 = idx(nd.d1_name);
                    nd.d2 = idx(nd.d2_name);
                }
                for (const auto& p : m.particles) g.particle_spin[idx(p.name)] = p.spin;
                for (const auto& nd : g.nodes) {
                    g.particle_spin[nd.mother] = nd.dj;
                    g.particle_spin[nd.d1] = nd.dj1;
                    g.particle_spin[nd.d2] = nd.dj2;
                }
                // momentum sources
                g.input_slot.assign(g.particle_names.size(), -3);
                g.sum_of.assign(g.particle_names.size(), {-1, -1});
                for (size_t i = 0; i < cfg.data_order.size(); ++i) g.input_slot[idx(cfg.data_order[i])] = (int)i;
                g.input_slot[idx(m.parent)] = -1;
                for (const auto& nd : g.nodes)
                    if (g.input_slot[nd.mother] == -3) {
                        g.input_slot[nd.mother] = -2;
                        g.sum_of[nd.mother] = {nd.d1, nd.d2};
                    }
                std::vector<bool> ready(g.particle_names.size(), false);
                for (size_t i = 0; i < ready.size(); ++i)
                    if (g.input_slot[i] >= 0) {
                        ready[i] = true;
                        g.build_order.push_back((int)i);
                    }
                for (size_t i = 0; i < ready.size(); ++i)
                    if (g.input_slot[i] == -1) {
                        ready[i] = true;
                        g.build_order.push_back((int)i);
                    }
                bool changed = true;
                while (changed) {
                    changed = false;
                    for (size_t i = 0; i < ready.size(); ++i)
                        if (!ready[i] && g.input_slot[i] == -2 && ready[g.sum_of[i].first] && ready[g.sum_of[i].second]) {
                            ready[i] = true;
                            g.build_order.push_back((int)i);
                            changed = true;
                        }
                }
                for (size_t i = 0; i < ready.size(); ++i)
                    if (!ready[i]) throw std::runtime_error("chain " + chain.name + ": cannot reconstruct momentum of " + g.particle_names[i]);
            }
            // SL combinations (src/AmpGen.cu:482-500)
            g.sl_combs = {{}};
            for (const auto& nd : g.nodes) {
                std::vector<std::vector<int>> t;
                for (const auto& c : g.sl_combs)
                    for (int s = 0; s < (int)nd.sls.size(); ++s) {
                        auto nc = c;
                        nc.push_back(s);
                        t.push_back(nc);
                    }
                g.sl_combs = std::move(t);
            }
            if (g.sl_combs.empty())
                m.cfg.warnings.push_back("chain \"" + chain.name + "\" has NO valid (S,L) wave combinations");
            // contraction label order (src/AmpGen.cu:1064-1185)
            {
                std::vector<int> labels;
                for (size_t ni = 0; ni < g.nodes.size(); ++ni) {
                    const auto& nd = g.nodes[ni];
                    if (ni == 0) {
                        labels = {nd.mother, nd.d1, nd.d2};
                        continue;
                    }
                    auto it = std::find(labels.begin(), labels.end(), nd.mother);
                    if (it == labels.end())
                        throw std::runtime_error("chain " + chain.name + ": mother " + nd.mother_name + " not produced by an earlier step");
                    labels.erase(it);
                    labels.push_back(nd.d1);
                    labels.push_back(nd.d2);
                }
                g.final_labels = labels;
                g.tensor_size = 1;
                for (int l : labels) g.tensor_size *= g.particle_spin[l];
                if (g.tensor_size != m.npol_total)
                    throw std::runtime_error("chain " + chain.name + ": final-state tensor does not cover all particles");
            }
            int gi = (int)m.groups.size();
            m.groups.push_back(g);
            const Group& G = m.groups.back();
            int nSL = G.nSL();

            // -- resonance combinations (src/Analysis.cu:4677-4720) --
            std::vector<std::vector<ResInstance>> rcombs = {{}};
            for (const auto& jp : comb) {
                const auto& rl = irmap[{jp.name, {jp.spin, jp.parity}}];
                std::vector<std::vector<ResInstance>> t;
                for (const auto& rc : rcombs)
                    for (const auto& r : rl) {
                        auto nc = rc;
                        nc.push_back(r);
                        t.push_back(nc);
                    }
                rcombs = std::move(t);
            }
            for (auto& rc : rcombs)
                for (auto& r : rc)
                    for (size_t pi = 0; pi < r.param_names.size(); ++pi) {
                        std::string nm = r.name + "_" + r.param_names[pi];
                        auto it = cfg.fix_var.find(nm);
                        if (it != cfg.fix_var.end() && !cfg.free_var.count(nm)) r.params[pi] = it->second;
                    }

            for (auto& rc : rcombs) {
                Block b;
                b.group = gi;
                b.site = gls;
                int bi = (int)m.blocks.size();
                for (auto& r : rc) {
                    r.particle_idx = (int)(std::lower_bound(G.particle_names.begin(), G.particle_names.end(), r.tag) -
                                           G.particle_names.begin());
                    r.node = -1;
                    for (size_t ni = 0; ni < G.nodes.size(); ++ni)
                        if (G.nodes[ni].mother_name == r.tag) {
                            r.node = (int)ni;
                            break;
                        }
                    // builtin AST settings (src/AmpGen.cu:2071-2101)
                    int Ldef = (r.type == ModelType::BWR) ? 1 : 2;
                    if (r.options.count("L")) Ldef = std::stoi(r.options["L"]);
                    r.d = r.options.count("d") ? std::stod(r.options["d"]) : 3.0;
                    r.has_bf = r.options.count("has_bf") ? (r.options["has_bf"] == "1" || r.options["has_bf"] == "true") : true;
                    r.Lmin = (r.node >= 0) ? G.nodes[r.node].l_min : Ldef;
                    if (r.node >= 0) {
                        const auto& nd = G.nodes[r.node];
                        const int didx[2] = {nd.d1, nd.d2};
                        for (int k = 0; k < 2; ++k) {
                            double ms = nd.mass[k + 1];
                            if (ms > 0) {
                                r.md_src[k] = MassSource::Fixed;
                                r.md_fixed[k] = ms;
                            } else if (didx[k] == r.particle_idx) {
                                r.md_src[k] = MassSource::M0Param;
                            } else {
                                r.md_src[k] = MassSource::Event;
                            }
                        }
                    }
                    r.theta.assign(r.params.size(), -1);
                }

                // free lists + trans skip (src/Analysis.cu:4728-4800)
                std::vector<std::vector<int>> all_free;
                std::vector<std::vector<std::vector<double>>> all_ranges;
                std::set<std::string> skip;
                std::map<std::string, std::string> conj_name;
                int ci = chain_comb_index[chain.name]++;
                for (size_t ri = 0; ri < rc.size(); ++ri) {
                    const auto& r = rc[ri];
                    auto it = cfg.resonances.find(r.name);
                    if (it != cfg.resonances.end() && !it->second.free.empty()) {
                        std::vector<int> fi;
                        if (it->second.free.size() == 1 && it->second.free[0] == -1) {
                            for (int pi = 0; pi < (int)r.param_names.size(); ++pi) fi.push_back(pi);
                        } else {
                            fi = it->second.free;
                        }
                        if (!cfg.fix_var.empty()) {
                            for (auto f = fi.begin(); f != fi.end();) {
                                std::string nm = (*f < (int)r.param_names.size()) ? r.name + "_" + r.param_names[*f]
                                                                                   : r.name + "_p" + std::to_string(*f);
                                if (cfg.fix_var.count(nm) && !cfg.free_var.count(nm)) f = fi.erase(f);
                                else ++f;
                            }
                        }
                        all_free.push_back(fi);
                        all_ranges.push_back(it->second.free_range);
                    } else {
                        all_free.push_back({});
                        all_ranges.push_back({});
                    }
                    if (!skip.count(r.name)) {
                        for (const auto& lc : chain_linked[chain.name]) {
                            auto lit = chain_resonances.find(lc);
                            if (lit != chain_resonances.end() && ci < (int)lit->second.size() &&
                                ri < lit->second[ci].size()) {
                                bool same = false;
                                for (const auto& per : lit->second)
                                    for (const auto& n : per)
                                        if (n == r.name) same = true;
                                if (same) break;
                                const std::string& owner = lit->second[ci][ri];
                                skip.insert(r.name);
                                if (r.name != owner) conj_name[r.name] = owner;
                                break;
                            }
                        }
                    }
                }
                {
                    std::vector<std::string> names;
                    for (const auto& r : rc) names.push_back(r.name);
                    auto& cr = chain_resonances[chain.name];
                    if (ci >= (int)cr.size()) cr.resize(ci + 1);
                    cr[ci] = names;
                }

                // theta slots (src/AmpGen.cu:2155-2210)
                for (size_t i = 0; i < rc.size(); ++i) {
                    if (skip.count(rc[i].name)) {
                        std::string owner = rc[i].name;
                        auto cn = conj_name.find(owner);
                        if (cn != conj_name.end()) owner = cn->second;
                        auto ow = resonance_owners.find(owner);
                        if (ow != resonance_owners.end()) conj_broadcast[{bi, (int)i}] = ow->second;
                        continue;
                    }
                    auto ow = resonance_owners.find(rc[i].name);
                    if (ow != resonance_owners.end() && !all_free[i].empty()) {
                        conj_broadcast[{bi, (int)i}] = ow->second;
                        continue;
                    }
                    resonance_owners[rc[i].name] = {bi, (int)i};
                    std::vector<int> exp;
                    if (!all_free[i].empty()) {
                        if (all_free[i].size() == 1 && all_free[i][0] == -1) {
                            for (int k = 0; k < (int)rc[i].params.size(); ++k) exp.push_back(k);
                        } else {
                            for (int k : all_free[i])
                                if (k >= 0 && k < (int)rc[i].params.size()) exp.push_back(k);
                        }
                    }
                    const auto& ranges = all_ranges[i];
                    for (size_t si = 0; si < exp.size(); ++si) {
                        int p = exp[si];
                        double val = rc[i].params[p];
                        double lo, hi;
                        if (si < ranges.size() && ranges[si].size() >= 2) {
                            lo = ranges[si][0];
                            hi = ranges[si][1];
                        } else {
                            double half = std::fabs(val) * 0.5;
                            lo = val - half;
                            hi = val + half;
                        }
                        std::string pname = p < (int)rc[i].param_names.size() ? rc[i].param_names[p] : "p" + std::to_string(p);
                        std::string sname = rc[i].name + "_" + pname;
                        auto vr = cfg.var_range.find(sname);
                        if (vr != cfg.var_range.end()) {
                            lo = vr->second.first;
                            hi = vr->second.second;
                        }
                        m.slots.push_back({bi, (int)i, p, val, lo, hi, sname});
                    }
                }
                b.res = rc;
                m.blocks.push_back(b);

                // amplitude names + coupling bookkeeping (src/Info.cu:205-320)
                auto rep = [&](const std::string& n) {
                    for (const auto& r : rc)
                        if (r.tag == n) return r.name;
                    return n;
                };
                std::string chain_key = chain.name;
                for (const auto& r : rc) chain_key += "_" + r.tag + "[" + r.name + "]";
                for (int s = 0; s < nSL; ++s) {
                    std::string full;
                    for (size_t ni = 0; ni < G.nodes.size(); ++ni) {
                        if (!full.empty()) full += "_";
                        const auto& nd = G.nodes[ni];
                        const SLPair& sl = nd.sls[G.sl_combs[s][ni]];
                        full += rep(nd.mother_name) + "→" + rep(nd.d1_name) + "+" + rep(nd.d2_name) + "_SL(" +
                                std::to_string(sl.S) + "," + std::to_string(sl.L) + ")";
                    }
                    amp_map.push_back({(int)m.amplitude_names.size(), chain_key});
                    m.amplitude_names.push_back(full);
                }
                gls += nSL;
            }
        }
    }

    // ---- var_equal (src/AmpGen.cu:2244-2342) ----
    struct Ghost {
        int block, res, param, owner;
    };
    std::vector<Ghost> ghosts;
    if (!cfg.var_equal.empty() && !m.slots.empty()) {
        std::map<std::string, int> n2s;
        for (size_t s = 0; s < m.slots.size(); ++s) n2s[m.slots[s].name] = (int)s;
        std::set<int> remove;
        struct Pending {
            Ghost g;
            int owner_pre;
        };
        std::vector<Pending> pend;
        for (const auto& grp : cfg.var_equal) {
            if (grp.size() < 2) continue;
            int owner = -1;
            for (const auto& n : grp) {
                auto it = n2s.find(n);
                if (it != n2s.end()) {
                    owner = it->second;
                    break;
                }
            }
            if (owner < 0 || remove.count(owner)) continue;
            for (const auto& n : grp) {
                auto it = n2s.find(n);
                if (it == n2s.end() || it->second == owner) continue;
                const auto& s = m.slots[it->second];
                pend.push_back({{s.block, s.res, s.param, -1}, owner});
                remove.insert(it->second);
            }
        }
        for (auto it = remove.rbegin(); it != remove.rend(); ++it) m.slots.erase(m.slots.begin() + *it);
        for (auto& p : pend) {
            int o = p.owner_pre;
            for (int r : remove)
                if (r < p.owner_pre) --o;
            p.g.owner = o;
            ghosts.push_back(p.g);
        }
    }

    // ---- theta sources per (block, res, param) ----
    for (size_t s = 0; s < m.slots.size(); ++s) {
        const auto& sl = m.slots[s];
        m.blocks[sl.block].res[sl.res].theta[sl.param] = (int)s;
    }
    for (const auto& g : ghosts) m.blocks[g.block].res[g.res].theta[g.param] = g.owner;
    // conjugate broadcast: all values of the owner resonance (src/AmpGen.cu:2468-2486)
    for (const auto& cb : conj_broadcast) {
        auto& cj = m.blocks[cb.first.first].res[cb.first.second];
        const auto& ow = m.blocks[cb.second.first].res[cb.second.second];
        size_t n = std::min(cj.params.size(), ow.params.size());
        for (size_t p = 0; p < n; ++p) {
            cj.params[p] = ow.params[p];
            cj.theta[p] = ow.theta[p];
        }
    }
    // per-call re-evaluation set (reference: block nFree > 0, incl. broadcast copies)
    std::vector<int> nfree(m.blocks.size(), 0);
    for (const auto& sl : m.slots) nfree[sl.block]++;
    for (const auto& g : ghosts) nfree[g.block]++;
    for (const auto& cb : conj_broadcast) nfree[cb.first.first] = std::max(nfree[cb.first.first], nfree[cb.second.first]);
    for (size_t b = 0; b < m.blocks.size(); ++b) m.blocks[b].free_path = nfree[b] > 0;

    // ---- coupling map: buildWithTrans (chain level) + vspace remap ----
    {
        int na = (int)m.amplitude_names.size();
        std::vector<std::string> keys;
        for (const auto& am : amp_map)
            if (std::find(keys.begin(), keys.end(), am.chain_key) == keys.end()) keys.push_back(am.chain_key);
        std::map<int, std::pair<int, double>> fold;
        for (const auto& c : cfg.constraints) {
            if (c.type != "trans" || c.names.size() < 2) continue;
            double ratio = c.values.empty() ? 1.0 : c.values[0].real();
            auto resName = [](const std::string& k) {
                auto p = k.rfind('[');
                return p != std::string::npos ? k.substr(p) : k;
            };
            std::map<std::string, int> A, B;
            for (size_t ci = 0; ci < keys.size(); ++ci) {
                if (keys[ci].find(c.names[0]) != std::string::npos) A[resName(keys[ci])] = (int)ci;
                if (keys[ci].find(c.names[1]) != std::string::npos) B[resName(keys[ci])] = (int)ci;
            }
            for (const auto& kb : B) {
                auto ia = A.find(kb.first);
                if (ia == A.end()) continue;
                fold[kb.second] = {ia->second, ratio};
            }
        }
        std::vector<std::string> active;
        for (size_t ci = 0; ci < keys.size(); ++ci)
            if (!fold.count((int)ci)) active.push_back(keys[ci]);
        std::vector<int> amp_chain(na, -1);
        std::vector<double> ratio(na, 1.0);
        for (const auto& am : amp_map) {
            int oc = (int)(std::find(keys.begin(), keys.end(), am.chain_key) - keys.begin());
            int fc = oc;
            double r = 1.0;
            if (fold.count(oc)) {
                fc = fold[oc].first;
                r = fold[oc].second;
            }
            amp_chain[am.amp_idx] = (int)(std::find(active.begin(), active.end(), keys[fc]) - active.begin());
            ratio[am.amp_idx] = r;
        }
        // vspace (src/Analysis.cu:4382-4478)
        std::map<int, std::vector<int>> owners;
        for (int a = 0; a < na; ++a)
            if (std::fabs(ratio[a] - 1.0) < 1e-10) owners[amp_chain[a]].push_back(a);
        bool split = false;
        for (const auto& o : owners)
            if (o.second.size() > 1) split = true;
        m.coupling.ratio = ratio;
        if (!split) {
            m.coupling.amp_chain = amp_chain;
            m.coupling.n_free = (int)active.size();
        } else {
            std::map<std::string, std::vector<int>> orig;
            for (const auto& am : amp_map) orig[am.chain_key].push_back(am.amp_idx);
            for (auto& kv : orig) std::sort(kv.second.begin(), kv.second.end());
            std::set<std::string> folded;
            for (const auto& kv : orig)
                if (!kv.second.empty() && std::fabs(ratio[kv.second[0]] - 1.0) > 1e-10) folded.insert(kv.first);
            int next = 0;
            std::map<int, std::vector<int>> acf;
            std::vector<int> ac2 = amp_chain;
            for (const auto& kv : orig) {
                if (folded.count(kv.first)) continue;
                int ac = amp_chain[kv.second[0]];
                for (int a : kv.second) {
                    ac2[a] = next;
                    acf[ac].push_back(next);
                    ++next;
                }
            }
            for (const auto& kv : orig) {
                if (!folded.count(kv.first)) continue;
                int ac = amp_chain[kv.second[0]];
                const auto& fi = acf[ac];
                for (size_t p = 0; p < kv.second.size() && p < fi.size(); ++p) ac2[kv.second[p]] = fi[p];
            }
            m.coupling.amp_chain = ac2;
            m.coupling.n_free = next;
        }
        std::map<int, std::string> f2n;
        for (int a = 0; a < na; ++a)
            if (std::fabs(m.coupling.ratio[a] - 1.0) < 1e-10) f2n[m.coupling.amp_chain[a]] = m.amplitude_names[a];
        for (const auto& kv : f2n) m.param_names.push_back(kv.second);
        for (const auto& s : m.slots) m.param_names.push_back(s.name);
    }

    addIdenticalVariants(cfg, m);

    // ---- gauss_constr (src/Analysis.cu:4003-4020) ----
    for (size_t s = 0; s < m.slots.size(); ++s) {
        auto it = cfg.gauss_constr.find(m.slots[s].name);
        if (it != cfg.gauss_constr.end()) m.gauss.push_back({(int)s, {m.slots[s].init, it->second}});
    }
    return m;
}

// ---------------------------------------------------------------------------
// JSON export
// ---------------------------------------------------------------------------
namespace {
std::string jstr(const std::string& s)
{
    std::string o = "\"";
    for (unsigned char c : s) {
        if (c == '"' || c == '\\') {
            o += '\\';
            o += (char)c;
        } else if (c < 0x20) {
            char buf[8];
            std::snprintf(buf, sizeof buf, "\\u%04x", c);
            o += buf;
        } else {
            o += (char)c;
        }
    }
    return o + "\"";
}
std::string jnum(double v)
{
    if (std::isnan(v)) return "null";
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    return buf;
}
template <class T, class F>
std::string jarr(const std::vector<T>& v, F f)
{
    std::string o = "[";
    for (size_t i = 0; i < v.size(); ++i) {
        if (i) o += ",";
        o += f(v[i]);
    }
    return o + "]";
}
std::string jint(int v) { return std::to_string(v); }
}  // namespace

std::string modelToJson(const Model& m)
{
    std::string o = "{";
    o += "\"npol\":" + jint(m.npol) + ",\"npol_total\":" + jint(m.npol_total);
    o += ",\"pol_map\":" + jarr(m.pol_map, jint);
    o += ",\"parent\":" + jstr(m.parent);
    o += ",\"final_order\":" + jarr(m.final_order, jstr);
    o += ",\"particles\":" + jarr(m.particles, [](const Particle& p) {
        return "{\"name\":" + jstr(p.name) + ",\"spin\":" + jint(p.spin) + ",\"parity\":" + jint(p.parity) +
               ",\"mass\":" + jnum(p.mass) + "}";
    });
    o += ",\"groups\":" + jarr(m.groups, [](const Group& g) {
        std::string s = "{\"chain\":" + jstr(g.chain_name);
        s += ",\"particles\":" + jarr(g.particle_names, jstr);
        s += ",\"spins\":" + jarr(g.particle_spin, jint);
        s += ",\"input_slot\":" + jarr(g.input_slot, jint);
        s += ",\"base\":" + jint(g.base) + ",\"sign\":" + jnum(g.sign) + ",\"variants\":" + jarr(g.variants, jint);
        s += ",\"sum_of\":" + jarr(g.sum_of, [](const std::pair<int, int>& p) {
            return "[" + jint(p.first) + "," + jint(p.second) + "]";
        });
        s += ",\"build_order\":" + jarr(g.build_order, jint);
        s += ",\"final_labels\":" + jarr(g.final_labels, jint);
        s += ",\"nodes\":" + jarr(g.nodes, [](const ModelNode& n) {
            return "{\"mother\":" + jint(n.mother) + ",\"d1\":" + jint(n.d1) + ",\"d2\":" + jint(n.d2) +
                   ",\"dj\":" + jint(n.dj) + ",\"dj1\":" + jint(n.dj1) + ",\"dj2\":" + jint(n.dj2) +
                   ",\"mass\":[" + jnum(n.mass[0]) + "," + jnum(n.mass[1]) + "," + jnum(n.mass[2]) + "]" +
                   ",\"has_bf\":" + (n.has_bf ? "true" : "false") + ",\"bf_d\":" + jnum(n.bf_d) +
                   ",\"l_min\":" + jint(n.l_min) + ",\"sls\":" +
                   jarr(n.sls, [](const SLPair& p) { return "[" + jint(p.S) + "," + jint(p.L) + "]"; }) + "}";
        });
        s += ",\"sl_combs\":" + jarr(g.sl_combs, [](const std::vector<int>& c) { return jarr(c, jint); });
        return s + "}";
    });
    o += ",\"blocks\":" + jarr(m.blocks, [](const Block& b) {
        std::string s = "{\"group\":" + jint(b.group) + ",\"site\":" + jint(b.site) +
                        ",\"free_path\":" + (b.free_path ? "true" : "false");
        s += ",\"res\":" + jarr(b.res, [](const ResInstance& r) {
            std::string t = "{\"name\":" + jstr(r.name) + ",\"tag\":" + jstr(r.tag) + ",\"type\":" +
                            jstr(modelTypeName(r.type)) + ",\"J\":" + jint(r.J) + ",\"P\":" + jint(r.P);
            t += ",\"params\":" + jarr(r.params, jnum);
            t += ",\"param_names\":" + jarr(r.param_names, jstr);
            t += ",\"theta\":" + jarr(r.theta, jint);
            t += ",\"channels\":" + jarr(r.channels, [](const std::pair<double, double>& c) {
                return "[" + jnum(c.first) + "," + jnum(c.second) + "]";
            });
            t += ",\"particle_idx\":" + jint(r.particle_idx) + ",\"node\":" + jint(r.node);
            t += ",\"Lmin\":" + jint(r.Lmin) + ",\"d\":" + jnum(r.d) + ",\"has_bf\":" + (r.has_bf ? "true" : "false");
            t += ",\"md_src\":[" + jint((int)r.md_src[0]) + "," + jint((int)r.md_src[1]) + "]";
            t += ",\"md_fixed\":[" + jnum(r.md_fixed[0]) + "," + jnum(r.md_fixed[1]) + "]";
            auto e = r.options.find("expr");
            t += ",\"expr\":" + (e != r.options.end() ? jstr(e->second) : std::string("null"));
            t += ",\"aux\":" + jarr(r.aux, jnum);
            return t + "}";
        });
        return s + "}";
    });
    o += ",\"amplitude_names\":" + jarr(m.amplitude_names, jstr);
    o += ",\"slots\":" + jarr(m.slots, [](const ThetaSlot& s) {
        return "{\"block\":" + jint(s.block) + ",\"res\":" + jint(s.res) + ",\"param\":" + jint(s.param) +
               ",\"init\":" + jnum(s.init) + ",\"lower\":" + jnum(s.lower) + ",\"upper\":" + jnum(s.upper) +
               ",\"name\":" + jstr(s.name) + "}";
    });
    o += ",\"coupling\":{\"n_free\":" + jint(m.coupling.n_free) + ",\"amp_chain\":" + jarr(m.coupling.amp_chain, jint) +
         ",\"ratio\":" + jarr(m.coupling.ratio, jnum) + "}";
    o += ",\"param_names\":" + jarr(m.param_names, jstr);
    o += ",\"gauss\":" + jarr(m.gauss, [](const std::pair<int, std::pair<double, double>>& g) {
        return "[" + jint(g.first) + "," + jnum(g.second.first) + "," + jnum(g.second.second) + "]";
    });
    o += ",\"warnings\":" + jarr(m.cfg.warnings, jstr);
    return o + "}";
}

}  // namespace ctpwa
