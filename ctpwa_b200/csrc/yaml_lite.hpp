// Minimal YAML reader for the ctpwa config.yml schema.
//
// The reference parses config.yml with yaml-cpp 0.8 (src/Config.cu:138-248).
// That library is not part of this build, so this file implements the subset
// of YAML 1.2 the schema uses:
//   - block mappings and block sequences (indentation based, '#' comments);
//   - flow sequences / flow mappings, nested, possibly spanning lines;
//   - single-pair flow mappings inside flow sequences ("[J: 1, P: -1]");
//   - complex (non-scalar) mapping keys such as "- [J: 1, P: -1]: [a, b]"
//     (yaml-cpp accepts these; PyYAML does not);
//   - plain, 'single' and "double" quoted scalars.
// Mappings keep insertion order, as yaml-cpp iteration does.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace ctpwa {
namespace yaml {

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

class Node {
public:
    enum class Kind { Null, Scalar, Seq, Map };

    Node() = default;
    static Node scalar(std::string s, bool quoted = false);
    static Node seq();
    static Node map();

    Kind kind() const { return kind_; }
    bool isNull() const { return kind_ == Kind::Null; }
    bool isScalar() const { return kind_ == Kind::Scalar; }
    bool isSeq() const { return kind_ == Kind::Seq; }
    bool isMap() const { return kind_ == Kind::Map; }
    // yaml-cpp's operator bool: a node that exists and is not null.
    explicit operator bool() const { return kind_ != Kind::Null; }

    // Sequence access.
    size_t size() const;
    const Node& operator[](size_t i) const;
    const Node& operator[](int i) const { return (*this)[(size_t)i]; }
    const std::vector<Node>& items() const { return items_; }
    void push(Node n) { items_.push_back(std::move(n)); }

    // Mapping access (scalar keys; a missing key yields a Null node).
    const Node& operator[](const std::string& key) const;
    const Node& operator[](const char* key) const { return (*this)[std::string(key)]; }
    const std::vector<std::pair<Node, Node>>& entries() const { return entries_; }
    void add(Node k, Node v) { entries_.emplace_back(std::move(k), std::move(v)); }

    // Scalar conversions (throw ParseError on mismatch).
    const std::string& str() const;
    double asDouble() const;
    int asInt() const;
    bool asBool() const;
    std::vector<std::string> asStrings() const;
    std::vector<double> asDoubles() const;
    std::vector<int> asInts() const;
    bool quoted() const { return quoted_; }

private:
    Kind kind_ = Kind::Null;
    bool quoted_ = false;
    std::string scalar_;
    std::vector<Node> items_;
    std::vector<std::pair<Node, Node>> entries_;
};

// Parse a whole document. Throws ParseError with a line number on failure.
Node parse(const std::string& text);
Node parseFile(const std::string& path);

}  // namespace yaml
}  // namespace ctpwa
