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
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <sstream>

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

Node readNode(std::istream& in, const std::string& path)
{
    std::string tag;
    if (!(in >> tag)) throw Exception("truncated node tree " + path);
    if (tag == "N") return Node::makeNull();
    std::size_t k = 0;
    if (!(in >> k)) throw Exception("malformed node tree " + path);
    if (tag == "S") {
        in.get();  // the newline after the length
        std::string s(k, '\0');
        in.read(&s[0], (std::streamsize)k);
        if ((std::size_t)in.gcount() != k) throw Exception("truncated scalar in " + path);
        return Node::makeScalar(s);
    }
    if (tag == "Q") {
        Node n = Node::makeSequence();
        for (std::size_t i = 0; i < k; ++i) n.push(readNode(in, path));
        return n;
    }
    if (tag == "M") {
        Node n = Node::makeMap();
        for (std::size_t i = 0; i < k; ++i) {
            Node key = readNode(in, path);
            Node val = readNode(in, path);
            n.insert(key, val);
        }
        return n;
    }
    throw Exception("unknown node tag '" + tag + "' in " + path);
}

}  // namespace

Node LoadFile(const std::string& path)
{
    {
        std::ifstream src(path);
        if (!src) throw BadFile(path);
    }
    const std::string tree = path + ".nodes";
    std::ifstream in(tree, std::ios::binary);
    if (!in) throw Exception("no composed node tree " + tree + " (write it with oracle/refcuda/yaml_nodes.py)");
    return readNode(in, tree);
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
    std::istringstream is(s);
    long long v = 0;
    is >> v;
    if (is.fail()) return false;
    is >> std::ws;
    if (!is.eof()) return false;
    *out = v;
    return true;
}

bool toDouble(const std::string& s, double* out)
{
    if (s == ".inf" || s == ".Inf" || s == ".INF" || s == "+.inf" || s == "+.Inf" || s == "+.INF")
        return (*out = std::numeric_limits<double>::infinity()), true;
    if (s == "-.inf" || s == "-.Inf" || s == "-.INF") return (*out = -std::numeric_limits<double>::infinity()), true;
    if (s == ".nan" || s == ".NaN" || s == ".NAN") return (*out = std::numeric_limits<double>::quiet_NaN()), true;
    std::istringstream is(s);
    double v = 0;
    is >> v;
    if (is.fail()) return false;
    is >> std::ws;
    if (!is.eof()) return false;
    *out = v;
    return true;
}

}  // namespace detail
}  // namespace YAML
