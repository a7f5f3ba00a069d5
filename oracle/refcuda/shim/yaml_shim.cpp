// ORACLE BUILD SHIM — test infrastructure, not product code.
// Implementation of the yaml-cpp subset of yaml-cpp/yaml.h over node trees
// composed by PyYAML (oracle/refcuda/yaml_nodes.py). Tree file format, one
// node in prefix order:
//   "S <n>\n" + n bytes + "\n"   scalar
//   "N\n"                        null
//   "Q <k>\n" + k nodes          sequence
//   "M <k>\n" + k (key, value)   mapping, document order
#include "yaml-cpp/yaml.h"

#include <cerrno>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <iterator>

namespace YAML {

Node::Node() : d_(std::make_shared<NodeData>()) {}

NodeType::value Node::Type() const { return d_ ? d_->type : NodeType::Undefined; }

const std::string& Node::Scalar() const
{
    static const std::string empty;
    return d_ && d_->type == NodeType::Scalar ? d_->scalar : empty;
}

std::size_t Node::size() const
{
    if (!d_) return 0;
    if (d_->type == NodeType::Sequence) return d_->seq.size();
    if (d_->type == NodeType::Map) return d_->map.size();
    return 0;
}

Node Node::operator[](const std::string& key) const
{
    if (d_ && d_->type == NodeType::Map)
        for (const auto& kv : d_->map)
            if (kv.first.IsScalar() && kv.first.Scalar() == key) return kv.second;
    return Node(nullptr, key);
}

Node Node::at(std::size_t index) const
{
    if (d_ && d_->type == NodeType::Sequence && index < d_->seq.size()) return d_->seq[index];
    return Node(nullptr, "[" + std::to_string(index) + "]");
}

const_iterator Node::begin() const { return const_iterator(d_, 0); }
const_iterator Node::end() const { return const_iterator(d_, size()); }

iterator_value const_iterator::operator*() const
{
    if (d_ && d_->type == NodeType::Sequence) return iterator_value(d_->seq[i_]);
    if (d_ && d_->type == NodeType::Map) return iterator_value(d_->map[i_].first, d_->map[i_].second);
    return iterator_value();
}

Node Node::makeScalar(const std::string& s)
{
    Node n;
    n.d_->type = NodeType::Scalar;
    n.d_->scalar = s;
    return n;
}
Node Node::makeNull() { return Node(); }
Node Node::makeSequence()
{
    Node n;
    n.d_->type = NodeType::Sequence;
    return n;
}
Node Node::makeMap()
{
    Node n;
    n.d_->type = NodeType::Map;
    return n;
}
void Node::push(const Node& n) { d_->seq.push_back(n); }
void Node::insert(const Node& k, const Node& v) { d_->map.emplace_back(k, v); }

namespace {

// The tree file is parsed by hand (no iostream number extraction, whose
// library implementation the host process may supply differently).
struct TreeReader {
    std::string buf;
    size_t at = 0;
    std::string path;

    [[noreturn]] void bad(const char* what) { throw Exception(std::string(what) + " in node tree " + path); }
    std::string word()
    {
        while (at < buf.size() && (buf[at] == ' ' || buf[at] == '\n')) ++at;
        size_t s = at;
        while (at < buf.size() && buf[at] != ' ' && buf[at] != '\n') ++at;
        if (s == at) bad("truncated");
        return buf.substr(s, at - s);
    }
    size_t count()
    {
        const std::string w = word();
        size_t v = 0;
        for (char c : w) {
            if (c < '0' || c > '9') bad("malformed count");
            v = v * 10 + (size_t)(c - '0');
        }
        return v;
    }
    Node node()
    {
        const std::string tag = word();
        if (tag == "N") return Node::makeNull();
        const size_t k = count();
        if (tag == "S") {
            if (at >= buf.size() || buf[at] != '\n') bad("malformed scalar");
            ++at;
            if (at + k > buf.size()) bad("truncated scalar");
            Node n = Node::makeScalar(buf.substr(at, k));
            at += k;
            return n;
        }
        if (tag == "Q") {
            Node n = Node::makeSequence();
            for (size_t i = 0; i < k; ++i) n.push(node());
            return n;
        }
        if (tag == "M") {
            Node n = Node::makeMap();
            for (size_t i = 0; i < k; ++i) {
                Node key = node();
                Node val = node();
                n.insert(key, val);
            }
            return n;
        }
        bad("unknown node tag");
    }
};

}  // namespace

Node LoadFile(const std::string& path)
{
    {
        std::ifstream src(path);
        if (!src) throw BadFile(path);
    }
    TreeReader r;
    r.path = path + ".nodes";
    std::ifstream in(r.path, std::ios::binary);
    if (!in) throw Exception("no composed node tree " + r.path + " (write it with oracle/refcuda/yaml_nodes.py)");
    r.buf.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
    return r.node();
}

namespace detail {

std::string scalarOf(const Node& n, const char* what)
{
    if (!n.IsScalar()) throw BadConversion(std::string("not a scalar (as ") + what + ")");
    return n.Scalar();
}

bool toBool(const std::string& s, bool* out)
{
    static const char* const yes[] = {"y", "Y", "yes", "Yes", "YES", "true", "True", "TRUE", "on", "On", "ON"};
    static const char* const no[] = {"n", "N", "no", "No", "NO", "false", "False", "FALSE", "off", "Off", "OFF"};
    for (const char* t : yes)
        if (s == t) return (*out = true), true;
    for (const char* t : no)
        if (s == t) return (*out = false), true;
    return false;
}

bool toLong(const std::string& s, long long* out)
{
    if (s.empty()) return false;
    const char* b = s.c_str();
    char* e = nullptr;
    errno = 0;
    const long long v = std::strtoll(b, &e, 10);
    if (e == b || errno) return false;
    while (*e == ' ' || *e == '\t') ++e;
    if (*e) return false;
    *out = v;
    return true;
}

bool toDouble(const std::string& s, double* out)
{
    if (s == ".inf" || s == ".Inf" || s == ".INF" || s == "+.inf" || s == "+.Inf" || s == "+.INF")
        return (*out = std::numeric_limits<double>::infinity()), true;
    if (s == "-.inf" || s == "-.Inf" || s == "-.INF") return (*out = -std::numeric_limits<double>::infinity()), true;
    if (s == ".nan" || s == ".NaN" || s == ".NAN") return (*out = std::numeric_limits<double>::quiet_NaN()), true;
    if (s.empty()) return false;
    const char* b = s.c_str();
    char* e = nullptr;
    const double v = std::strtod(b, &e);
    if (e == b) return false;
    while (*e == ' ' || *e == '\t') ++e;
    if (*e) return false;
    *out = v;
    return true;
}

}  // namespace detail
}  // namespace YAML
