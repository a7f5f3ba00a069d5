// ORACLE BUILD SHIM — test infrastructure, not product code.
//
// The subset of the yaml-cpp 0.8 interface that the reference's config
// reader uses (src/Config.cu, include/Config.cuh:8), so that the reference
// builds unmodified where yaml-cpp is not installed. The document is not
// parsed here: YAML::LoadFile(path) reads the node tree that PyYAML composed
// from `path` (oracle/refcuda/yaml_nodes.py writes it to `path + ".nodes"`),
// so the YAML grammar itself comes from an independent implementation.
// Semantics follow yaml-cpp: operator[] on a missing key gives an undefined
// node that converts to false; as<T>() on an undefined node throws
// InvalidNode and on a wrong type or text throws BadConversion; maps keep
// document order when iterated.
#pragma once

#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace YAML {

class Exception : public std::runtime_error {
public:
    explicit Exception(const std::string& m) : std::runtime_error(m), msg(m) {}
    std::string msg;
};
class BadFile : public Exception {
public:
    explicit BadFile(const std::string& f) : Exception("bad file: " + f) {}
};
class InvalidNode : public Exception {
public:
    explicit InvalidNode(const std::string& k) : Exception("invalid node; this may result from using a map iterator as a sequence iterator, or vice-versa (key: " + k + ")") {}
};
class BadConversion : public Exception {
public:
    explicit BadConversion(const std::string& m) : Exception("bad conversion: " + m) {}
};

namespace NodeType {
enum value { Undefined, Null, Scalar, Sequence, Map };
}

class Node;
struct NodeData;

class iterator_value;
class const_iterator;

class Node {
public:
    Node();
    NodeType::value Type() const;
    bool IsDefined() const { return Type() != NodeType::Undefined; }
    bool IsNull() const { return Type() == NodeType::Null; }
    bool IsScalar() const { return Type() == NodeType::Scalar; }
    bool IsSequence() const { return Type() == NodeType::Sequence; }
    bool IsMap() const { return Type() == NodeType::Map; }
    explicit operator bool() const { return IsDefined(); }
    bool operator!() const { return !IsDefined(); }
    const std::string& Scalar() const;
    std::size_t size() const;

    Node operator[](const std::string& key) const;
    Node operator[](const char* key) const { return (*this)[std::string(key)]; }
    Node operator[](int index) const { return at((std::size_t)(index < 0 ? (std::size_t)-1 : (std::size_t)index)); }
    Node operator[](std::size_t index) const { return at(index); }

    template <class T>
    T as() const;
    template <class T, class S>
    T as(const S& fallback) const
    {
        if (!IsDefined()) return fallback;
        try {
            return as<T>();
        } catch (const Exception&) {
            return fallback;
        }
    }

    const_iterator begin() const;
    const_iterator end() const;

    // tree construction (used by the reader)
    static Node makeScalar(const std::string& s);
    static Node makeNull();
    static Node makeSequence();
    static Node makeMap();
    void push(const Node& n);
    void insert(const Node& k, const Node& v);

private:
    explicit Node(std::shared_ptr<NodeData> d, std::string key = "") : d_(std::move(d)), key_(std::move(key)) {}
    Node at(std::size_t index) const;
    std::shared_ptr<NodeData> d_;  // null: undefined
    std::string key_;              // the key this node was looked up by (messages)
    friend class const_iterator;
};

struct NodeData {
    NodeType::value type = NodeType::Null;
    std::string scalar;
    std::vector<Node> seq;
    std::vector<std::pair<Node, Node>> map;
};

// What iterating a node yields: for a sequence the element (this node), for a
// map the pair (first, second).
class iterator_value : public Node, public std::pair<Node, Node> {
public:
    iterator_value() {}
    explicit iterator_value(const Node& n) : Node(n) {}
    iterator_value(const Node& k, const Node& v) : Node(), std::pair<Node, Node>(k, v) {}
};

class const_iterator {
public:
    const_iterator(std::shared_ptr<NodeData> d, std::size_t i) : d_(std::move(d)), i_(i) {}
    iterator_value operator*() const;
    std::unique_ptr<iterator_value> operator->() const { return std::unique_ptr<iterator_value>(new iterator_value(**this)); }
    const_iterator& operator++()
    {
        ++i_;
        return *this;
    }
    bool operator==(const const_iterator& o) const { return d_ == o.d_ && i_ == o.i_; }
    bool operator!=(const const_iterator& o) const { return !(*this == o); }

private:
    std::shared_ptr<NodeData> d_;
    std::size_t i_;
};
using iterator = const_iterator;

Node LoadFile(const std::string& path);

// conversions
namespace detail {
std::string scalarOf(const Node& n, const char* what);
bool toBool(const std::string& s, bool* out);
bool toLong(const std::string& s, long long* out);
bool toDouble(const std::string& s, double* out);
}  // namespace detail

template <class T>
struct convert;

template <>
struct convert<std::string> {
    static std::string decode(const Node& n) { return detail::scalarOf(n, "string"); }
};
template <>
struct convert<bool> {
    static bool decode(const Node& n)
    {
        bool b = false;
        if (!detail::toBool(detail::scalarOf(n, "bool"), &b)) throw BadConversion("not a boolean: " + n.Scalar());
        return b;
    }
};
template <>
struct convert<int> {
    static int decode(const Node& n)
    {
        long long v = 0;
        if (!detail::toLong(detail::scalarOf(n, "int"), &v)) throw BadConversion("not an integer: " + n.Scalar());
        return (int)v;
    }
};
template <>
struct convert<long> {
    static long decode(const Node& n)
    {
        long long v = 0;
        if (!detail::toLong(detail::scalarOf(n, "long"), &v)) throw BadConversion("not an integer: " + n.Scalar());
        return (long)v;
    }
};
template <>
struct convert<double> {
    static double decode(const Node& n)
    {
        double v = 0;
        if (!detail::toDouble(detail::scalarOf(n, "double"), &v)) throw BadConversion("not a number: " + n.Scalar());
        return v;
    }
};
template <>
struct convert<float> {
    static float decode(const Node& n) { return (float)convert<double>::decode(n); }
};
template <class T>
struct convert<std::vector<T>> {
    static std::vector<T> decode(const Node& n)
    {
        if (!n.IsDefined()) throw InvalidNode("sequence");
        if (!n.IsSequence()) throw BadConversion("not a sequence");
        std::vector<T> out;
        for (std::size_t i = 0; i < n.size(); ++i) out.push_back(convert<T>::decode(n[i]));
        return out;
    }
};

template <class T>
T Node::as() const
{
    if (!IsDefined()) throw InvalidNode(key_);
    return convert<T>::decode(*this);
}

}  // namespace YAML
