// config.yml schema -> Config (see config.hpp for the reference mapping).
#include "config.hpp"

#include "yaml_lite.hpp"

#include <cmath>
#include <filesystem>
#include <fstream>
#include <queue>
#include <sstream>
#include <stdexcept>

namespace ctpwa {

using yaml::Node;

const Particle* Config::findParticle(const std::string& n) const
{
    for (const auto& p : particles)
        if (p.name == n) return &p;
    return nullptr;
}

float transJValue(const std::string& s)
{
    size_t slash = s.find('/');
    if (slash != std::string::npos) {
        float num = std::stof(s.substr(0, slash));
        float den = std::stof(s.substr(slash + 1));
        return den != 0.0f ? num / den : 0.0f;
    }
    std::stringstream ss(s);
    float v;
    if (ss >> v) return v;
    return 0.0f;
}

namespace {

std::string trimS(const std::string& s)
{
    size_t b = s.find_first_not_of(" \t\r\n");
    if (b == std::string::npos) return "";
    size_t e = s.find_last_not_of(" \t\r\n");
    return s.substr(b, e - b + 1);
}

int spinOf(const Node& n) { return (int)(2.0f * transJValue(n.str()) + 1.0f); }

// [S, L] or [[S1, L1], ...] with S a physical spin -> {2S+1, L}
// (src/Config.cu:620-633, 761-775)
std::vector<std::vector<int>> parseSlFilterPhysical(const Node& sl)
{
    std::vector<std::vector<int>> out;
    std::vector<std::vector<double>> raw;
    if (sl[0].isSeq()) {
        for (const auto& row : sl.items()) raw.push_back(row.asDoubles());
    } else {
        raw.push_back(sl.asDoubles());
    }
    for (const auto& row : raw)
        if (row.size() >= 2) out.push_back({(int)std::lround(2.0 * row[0] + 1.0), (int)row[1]});
    return out;
}

void parseParticles(Config& c, const Node& node)
{
    for (const auto& kv : node.entries()) {
        Particle p;
        p.name = kv.first.str();
        const Node& props = kv.second;
        p.spin = spinOf(props["J"]);
        p.parity = props["P"].asInt();
        p.mass = props["mass"].asDouble();
        if (props["polarization"] && props["polarization"].isSeq())
            for (const auto& m : props["polarization"].items())
                p.polarization_2m.push_back((int)(2.0f * transJValue(m.str())));
        c.particles.push_back(p);
    }
}

void parseData(Config& c, const Node& node)
{
    if (node["order"]) c.data_order = node["order"].asStrings();
    for (const char* k : {"data", "phsp", "phsp_truth", "bkg", "bkg_weights", "data_weights", "phsp_weights"})
        if (node[k]) c.data_files[k] = node[k].asStrings();
}

void parseResonances(Config& c, const Node& node)
{
    for (const auto& kv : node.entries()) {
        ResonanceConfig r;
        r.name = kv.first.str();
        const Node& props = kv.second;
        r.J = props["J"] ? spinOf(props["J"]) : -1;
        r.P = props["P"] ? props["P"].asInt() : 0;
        if (!props["model"]) throw std::runtime_error("resonance '" + r.name + "' has no model");
        r.type = props["model"].str();
        if (props["paramValues"]) r.parameters = props["paramValues"].asDoubles();
        else if (props["parameters"]) r.parameters = props["parameters"].asDoubles();
        if (props["file"]) r.options["file"] = props["file"].str();
        if (props["bins"]) r.options["bins"] = props["bins"].str();
        if (props["range"]) {
            auto rg = props["range"].asDoubles();
            std::string s;
            for (size_t i = 0; i < rg.size(); ++i) {
                if (i) s += ",";
                s += std::to_string(rg[i]);
            }
            r.options["range"] = s;
        }
        if (props["extrapolate"]) r.options["extrapolate"] = props["extrapolate"].str();
        const Node& pn = props["paramNames"] ? props["paramNames"] : props["params"];
        if (pn) {
            auto pl = pn.asStrings();
            std::string s;
            for (size_t i = 0; i < pl.size(); ++i) {
                if (i) s += ",";
                s += pl[i];
            }
            r.options["params"] = s;
        }
        if (props["expr"]) r.options["expr"] = props["expr"].str();
        if (props["channels"])
            for (const auto& ch : props["channels"].items()) r.channels.push_back(ch.asDoubles());
        if (props["free"]) r.free = props["free"].asInts();
        if (props["has_bf"]) {
            r.has_bf = props["has_bf"].asBool();
            r.has_bf_explicit = true;
        }
        if (props["bf_d"]) r.bf_d = props["bf_d"].asDouble();
        if (props["free_range"])
            for (const auto& rn : props["free_range"].items()) r.free_range.push_back(rn.asDoubles());
        c.resonances[r.name] = r;
    }
}

// Explicit [J: .., P: ..] key of an intermediates entry -> {2J+1, P}
std::vector<int> parseJPKey(const Node& key)
{
    std::vector<int> sp;
    if (!key.isSeq()) return sp;
    for (const auto& jp : key.items()) {
        if (jp["J"]) sp.push_back((int)(2.0f * transJValue(jp["J"].str()) + 1.0f));
        if (jp["P"]) sp.push_back(jp["P"].asInt());
    }
    return sp;
}

struct IntDecay {
    std::string d1, d2;
    bool has_bf = true;
    bool has_bf_explicit = false;
    double bf_d = NAN;
    bool p_break = false;
    std::vector<std::vector<int>> sl_filter;
};

IntDecay parseOneMode(const Node& n)
{
    IntDecay id;
    id.d1 = n[0].str();
    id.d2 = n[1].str();
    if (n.size() >= 3 && n[2].isMap()) {
        const Node& o = n[2];
        if (o["has_bf"]) {
            id.has_bf = o["has_bf"].asBool();
            id.has_bf_explicit = true;
        }
        if (o["bf_d"]) id.bf_d = o["bf_d"].asDouble();
        if (o["p_break"]) id.p_break = o["p_break"].asBool();
        if (o["sl"]) id.sl_filter = parseSlFilterPhysical(o["sl"]);
    }
    return id;
}

// Compact chain block -> one or more DecayChainConfig (src/Config.cu:590-951)
void expandCompactChain(Config& c, const std::string& chain_name, const Node& chain_data,
                        const std::string& mother)
{
    const Node& channels = chain_data[mother];

    std::map<std::string, std::vector<IntDecay>> modes;
    for (const auto& kv : chain_data.entries()) {
        std::string key = kv.first.str();
        if (key == mother || key == "intermediates" || key == "legend" || key == "symmetrize") continue;
        if (!kv.second.isSeq() || kv.second.size() == 0) continue;
        if (kv.second[0].isSeq()) {
            for (const auto& m : kv.second.items()) modes[key].push_back(parseOneMode(m));
        } else if (kv.second.size() >= 2 && kv.second[0].isScalar()) {
            modes[key].push_back(parseOneMode(kv.second));
        }
    }
    auto getMode = [&](const std::string& name, size_t idx) -> const IntDecay* {
        auto it = modes.find(name);
        if (it == modes.end() || idx >= it->second.size()) return nullptr;
        return &it->second[idx];
    };

    std::map<std::string, ResonanceChainConfig> res_chain_map;
    if (chain_data["intermediates"]) {
        for (const auto& rn : chain_data["intermediates"].entries()) {
            ResonanceChainConfig rc;
            rc.intermediate = rn.first.str();
            for (const auto& spin_node : rn.second.items()) {
                if (spin_node.isMap()) {
                    for (const auto& sp : spin_node.entries()) {
                        SpinChainConfig sc;
                        sc.spin_parity = parseJPKey(sp.first);
                        sc.resonances = sp.second.asStrings();
                        rc.spin_chains.push_back(sc);
                    }
                } else if (spin_node.isSeq()) {
                    // Auto-detect form: group the listed resonances by (J, P).
                    std::map<std::pair<int, int>, std::vector<std::string>> groups;
                    for (const auto& rnm : spin_node.items()) {
                        std::string name = rnm.str();
                        auto it = c.resonances.find(name);
                        if (it == c.resonances.end()) {
                            c.warnings.push_back("resonance '" + name + "' not found in Resonances section");
                            continue;
                        }
                        if (it->second.J < 0)
                            throw std::runtime_error("resonance without J/P requires explicit [J,P] form: " + name);
                        groups[{it->second.J, it->second.P}].push_back(name);
                    }
                    for (const auto& g : groups) {
                        SpinChainConfig sc;
                        sc.spin_parity = {g.first.first, g.first.second};
                        sc.resonances = g.second;
                        rc.spin_chains.push_back(sc);
                    }
                }
            }
            res_chain_map[rc.intermediate] = rc;
        }
    }

    for (const auto& ch : channels.items()) {
        std::string bachelor = ch[0].str();
        std::string intermediate = ch[1].str();

        bool has_bf1 = true, has_bf2 = true, has_bf1_x = false, has_bf2_x = false;
        double bf_d1 = NAN, bf_d2 = NAN;
        bool pb1 = false, pb2 = false, has_pb = false;
        std::vector<std::vector<int>> sl1;
        if (ch.size() >= 3 && ch[2].isMap()) {
            const Node& o = ch[2];
            if (o["has_bf"]) {
                if (o["has_bf"].isSeq()) {
                    has_bf1 = o["has_bf"][0].asBool();
                    has_bf2 = o["has_bf"][1].asBool();
                } else {
                    has_bf1 = has_bf2 = o["has_bf"].asBool();
                }
                has_bf1_x = has_bf2_x = true;
            }
            if (o["bf_d"]) {
                if (o["bf_d"].isSeq()) {
                    bf_d1 = o["bf_d"][0].asDouble();
                    bf_d2 = o["bf_d"][1].asDouble();
                } else {
                    bf_d1 = bf_d2 = o["bf_d"].asDouble();
                }
            }
            if (o["p_break"]) {
                has_pb = true;
                if (o["p_break"].isSeq()) {
                    pb1 = o["p_break"][0].asBool();
                    pb2 = o["p_break"][1].asBool();
                } else {
                    pb1 = pb2 = o["p_break"].asBool();
                }
            }
            if (o["sl"]) sl1 = parseSlFilterPhysical(o["sl"]);
        }

        size_t n_modes = 1;
        bool bachelor_drives = false;
        if (modes.count(intermediate)) {
            n_modes = modes[intermediate].size();
        } else if (modes.count(bachelor)) {
            n_modes = modes[bachelor].size();
            bachelor_drives = true;
        }

        for (size_t mi = 0; mi < n_modes; ++mi) {
            if (n_modes > 1) {
                const IntDecay* m = bachelor_drives ? getMode(bachelor, mi) : getMode(intermediate, mi);
                const std::string& other = bachelor_drives ? intermediate : bachelor;
                if (m && (m->d1 == other || m->d2 == other)) continue;
            }
            DecayChainConfig chain;
            chain.name = chain_name + "_" + (bachelor_drives ? bachelor : intermediate);
            if (n_modes > 1) chain.name += "_" + std::to_string(mi);

            DecayStep s1;
            s1.mother = mother;
            s1.daughters = {bachelor, intermediate};
            s1.has_bf = has_bf1;
            s1.has_bf_explicit = has_bf1_x;
            s1.bf_d = bf_d1;
            s1.p_break = pb1;
            s1.sl_filter = sl1;
            chain.decay_steps.push_back(s1);

            bool int_decays = modes.count(intermediate) > 0;
            bool bach_decays = modes.count(bachelor) > 0;
            if (!int_decays && res_chain_map.count(intermediate))
                chain.resonance_chains.push_back(res_chain_map[intermediate]);
            if (!bach_decays && res_chain_map.count(bachelor))
                chain.resonance_chains.push_back(res_chain_map[bachelor]);
            if (!int_decays && !bach_decays) {
                c.decay_chains.push_back(chain);
                continue;
            }

            struct Item {
                std::string name;
                bool is_first;
                bool has_bf, has_bf_x, pb;
                double bf_d;
                std::vector<std::vector<int>> sl;
            };
            std::queue<Item> q;
            if (int_decays) {
                const IntDecay* ifm = getMode(intermediate, bachelor_drives ? 0 : mi);
                bool hb = has_bf2_x ? has_bf2 : (ifm && ifm->has_bf_explicit ? ifm->has_bf : true);
                bool hbx = has_bf2_x || (ifm && ifm->has_bf_explicit);
                double bd = !std::isnan(bf_d2) ? bf_d2 : (ifm && !std::isnan(ifm->bf_d) ? ifm->bf_d : NAN);
                bool pb = has_pb ? pb2 : (ifm ? ifm->p_break : false);
                q.push({intermediate, !bachelor_drives, hb, hbx, pb, bd,
                        ifm ? ifm->sl_filter : std::vector<std::vector<int>>{}});
            }
            if (bach_decays) {
                const IntDecay* bm = getMode(bachelor, bachelor_drives ? mi : 0);
                q.push({bachelor, bachelor_drives, bm && bm->has_bf_explicit ? bm->has_bf : true,
                        bm && bm->has_bf_explicit, bm ? bm->p_break : false,
                        (bm && !std::isnan(bm->bf_d)) ? bm->bf_d : NAN,
                        bm ? bm->sl_filter : std::vector<std::vector<int>>{}});
            }
            while (!q.empty()) {
                Item it = q.front();
                q.pop();
                const IntDecay* mode = getMode(it.name, it.is_first ? mi : 0);
                if (!mode) continue;
                DecayStep st;
                st.mother = it.name;
                st.daughters = {mode->d1, mode->d2};
                st.has_bf = it.has_bf;
                st.has_bf_explicit = it.has_bf_x;
                st.bf_d = it.bf_d;
                st.p_break = it.pb;
                st.sl_filter = it.sl;
                chain.decay_steps.push_back(st);
                if (res_chain_map.count(it.name)) chain.resonance_chains.push_back(res_chain_map[it.name]);
                for (const std::string& d : {mode->d1, mode->d2}) {
                    if (modes.count(d)) {
                        const IntDecay* dm = getMode(d, 0);
                        q.push({d, false, dm && dm->has_bf_explicit ? dm->has_bf : true,
                                dm && dm->has_bf_explicit, dm ? dm->p_break : false,
                                (dm && !std::isnan(dm->bf_d)) ? dm->bf_d : NAN,
                                dm ? dm->sl_filter : std::vector<std::vector<int>>{}});
                    }
                }
            }
            c.decay_chains.push_back(chain);
        }
    }
}

// Expanded chain block (src/Config.cu:953-1036)
void parseExpandedChain(Config& c, const std::string& chain_name, const Node& chain_data)
{
    DecayChainConfig chain;
    chain.name = chain_name;
    if (chain_data["decay"]) {
        for (const auto& step_node : chain_data["decay"].items()) {
            for (const auto& dp : step_node.entries()) {
                DecayStep st;
                st.mother = dp.first.str();
                if (dp.second.isSeq()) {
                    st.daughters = dp.second.asStrings();
                } else if (dp.second.isMap()) {
                    const Node& o = dp.second;
                    st.daughters = o["daughters"].asStrings();
                    if (o["has_bf"]) {
                        st.has_bf = o["has_bf"].asBool();
                        st.has_bf_explicit = true;
                    }
                    if (o["bf_d"]) st.bf_d = o["bf_d"].asDouble();
                    if (o["p_break"]) st.p_break = o["p_break"].asBool();
                    if (o["sl"]) {
                        // expanded form: S given in 2S+1 notation already
                        if (o["sl"][0].isSeq())
                            for (const auto& row : o["sl"].items()) st.sl_filter.push_back(row.asInts());
                        else
                            st.sl_filter.push_back(o["sl"].asInts());
                    }
                }
                chain.decay_steps.push_back(st);
            }
        }
    }
    for (const auto& rn : chain_data.entries()) {
        std::string key = rn.first.str();
        if (key == "decay" || key == "legend" || key == "symmetrize") continue;
        ResonanceChainConfig rc;
        rc.intermediate = key;
        for (const auto& spin_node : rn.second.items()) {
            for (const auto& sp : spin_node.entries()) {
                SpinChainConfig sc;
                sc.spin_parity = parseJPKey(sp.first);
                sc.resonances = sp.second.asStrings();
                rc.spin_chains.push_back(sc);
            }
        }
        chain.resonance_chains.push_back(rc);
    }
    c.decay_chains.push_back(chain);
}

void parseDecayChains(Config& c, const Node& node)
{
    std::set<std::string> pnames;
    for (const auto& p : c.particles) pnames.insert(p.name);
    for (const auto& kv : node.entries()) {
        std::string chain_name = kv.first.str();
        const Node& cd = kv.second;
        std::string mother;
        bool compact = false;
        if (!cd["decay"]) {
            for (const auto& e : cd.entries()) {
                if (!e.first.isScalar()) continue;
                std::string key = e.first.str();
                if (key == "intermediates" || key == "legend" || key == "symmetrize") continue;
                if (pnames.count(key) && e.second.isSeq() && e.second.size() > 0 &&
                    e.second[0].isSeq() && e.second[0].size() >= 2) {
                    mother = key;
                    compact = true;
                    break;
                }
            }
        }
        if (compact) expandCompactChain(c, chain_name, cd, mother);
        else parseExpandedChain(c, chain_name, cd);
    }
}

void parseIdentical(Config& c, const Node& ident)
{
    int gi = 1;
    for (const auto& g : ident.items()) {
        auto names = g.asStrings();
        std::string gname = "identical" + std::to_string(gi++);
        for (auto& p : c.particles)
            for (const auto& n : names)
                if (p.name == n) p.identical_group = gname;
    }
}

void parseConstraints(Config& c, const Node& node)
{
    c.constraints.clear();
    if (node["maxL"]) c.global_maxL = node["maxL"].asInt();
    if (node["bf_d"]) c.global_bf_d = node["bf_d"].asDouble();
    if (node["has_bf"]) c.global_has_bf = node["has_bf"].asBool();
    if (node["fix_var"])
        for (const auto& kv : node["fix_var"].entries()) c.fix_var[kv.first.str()] = kv.second.asDouble();
    if (node["free_var"])
        for (const auto& n : node["free_var"].items()) c.free_var.insert(n.str());
    if (node["var_range"]) {
        for (const auto& kv : node["var_range"].entries()) {
            if (kv.second.isSeq() && kv.second.size() >= 2)
                c.var_range[kv.first.str()] = {kv.second[0].asDouble(), kv.second[1].asDouble()};
            else
                c.warnings.push_back("var_range entry '" + kv.first.str() + "' ignored (needs [lower, upper])");
        }
    }
    if (node["var_equal"]) {
        for (const auto& g : node["var_equal"].items()) {
            auto names = g.asStrings();
            if (names.size() >= 2) c.var_equal.push_back(names);
        }
    }
    if (node["gauss_constr"])
        for (const auto& kv : node["gauss_constr"].entries()) c.gauss_constr[kv.first.str()] = kv.second.asDouble();
    if (node["identical"]) parseIdentical(c, node["identical"]);
    if (node["trans"]) {
        for (const auto& lst : node["trans"].items()) {
            for (const auto& pr : lst.entries()) {
                ConstraintConfig cc;
                cc.type = "trans";
                cc.names = pr.first.asStrings();
                const Node& v = pr.second;
                if (v.isSeq()) {
                    if (v.size() > 0 && v[0].isSeq()) {
                        for (const auto& row : v.items())
                            if (row.isSeq() && row.size() >= 2)
                                cc.values.emplace_back(row[0].asDouble(), row[1].asDouble());
                    } else {
                        for (const auto& x : v.items()) cc.values.emplace_back(x.asDouble(), 0.0);
                    }
                } else if (v.isScalar()) {
                    cc.values.emplace_back(v.asDouble(), 0.0);
                }
                c.constraints.push_back(cc);
            }
        }
    }
}

// per-step > resonance (mother) > Constraints global > default (src/Config.cu:1140-1176)
void resolveStepBF(Config& c)
{
    for (auto& chain : c.decay_chains) {
        for (auto& step : chain.decay_steps) {
            const ResonanceConfig* cfg = nullptr;
            auto it = c.resonances.find(step.mother);
            if (it != c.resonances.end()) {
                cfg = &it->second;
            } else {
                for (const auto& rc : chain.resonance_chains) {
                    if (rc.intermediate != step.mother || rc.spin_chains.empty()) continue;
                    const auto& rn = rc.spin_chains[0].resonances;
                    if (!rn.empty()) {
                        auto rit = c.resonances.find(rn[0]);
                        if (rit != c.resonances.end()) cfg = &rit->second;
                    }
                    break;
                }
            }
            if (!step.has_bf_explicit) step.has_bf = (cfg && cfg->has_bf_explicit) ? cfg->has_bf : c.global_has_bf;
            if (std::isnan(step.bf_d)) step.bf_d = (cfg && !std::isnan(cfg->bf_d)) ? cfg->bf_d : c.global_bf_d;
        }
    }
}

std::filesystem::path dirOf(const std::string& path)
{
    return std::filesystem::path(path).parent_path();
}

}  // namespace

Config loadConfigText(const std::string& text, const std::string& path)
{
    Config c;
    c.config_file = path;
    Node root;
    try {
        root = yaml::parse(text);
    } catch (const yaml::ParseError& e) {
        c.warnings.push_back(std::string("failed to parse config: ") + e.what());
        return c;  // invalid (no particles)
    }
    if (!root.isMap()) return c;

    if (root["Particles"]) parseParticles(c, root["Particles"]);
    if (root["Data"]) parseData(c, root["Data"]);
    const Node& cons = root["Constraints"];
    if (cons && cons["identical"]) parseIdentical(c, cons["identical"]);
    if (cons && cons["chains"]) {
        const Node& ch = cons["chains"];
        if (ch.isScalar()) {
            std::ifstream f(dirOf(path) / ch.str());
            std::string line;
            while (std::getline(f, line)) {
                std::string pat = trimS(line);
                if (pat.empty() || pat[0] == '#') continue;
                c.chain_filter.push_back(pat);
            }
            if (c.chain_filter.empty()) c.warnings.push_back("chain filter file empty or not found");
        } else if (ch.isSeq()) {
            c.chain_filter = ch.asStrings();
        }
    }
    if (root["Resonances"]) {
        if (root["Resonances"].isScalar()) {
            auto rp = dirOf(path) / root["Resonances"].str();
            try {
                Node rn = yaml::parseFile(rp.string());
                if (rn["Resonances"]) rn = Node(rn["Resonances"]);
                parseResonances(c, rn);
            } catch (const yaml::ParseError& e) {
                c.warnings.push_back("failed to load external resonance file " + rp.string() + ": " + e.what());
            }
        } else {
            parseResonances(c, root["Resonances"]);
        }
    }
    if (root["DecayChains"]) parseDecayChains(c, root["DecayChains"]);
    if (cons) parseConstraints(c, cons);
    resolveStepBF(c);
    if (root["precision"]) c.precision = root["precision"].str();
    if (!c.chain_filter.empty() && !c.decay_chains.empty()) {
        std::vector<DecayChainConfig> kept;
        for (const auto& dc : c.decay_chains)
            for (const auto& pat : c.chain_filter)
                if (dc.name.find(pat) != std::string::npos) {
                    kept.push_back(dc);
                    break;
                }
        c.decay_chains = std::move(kept);
    }
    return c;
}

Config loadConfig(const std::string& path)
{
    std::ifstream f(path);
    if (!f.is_open()) {
        Config c;
        c.config_file = path;
        c.warnings.push_back("config file not found: " + path);
        return c;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    return loadConfigText(ss.str(), path);
}

}  // namespace ctpwa
