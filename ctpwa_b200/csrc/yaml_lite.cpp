// Minimal YAML reader for the ctpwa config.yml schema (see yaml_lite.hpp).
#include "yaml_lite.hpp"

#include <cctype>
#include <cerrno>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace ctpwa {
namespace yaml {

namespace {
const Node& nullNode()
{
    static const Node n;
    return n;
}
}  // namespace

Node Node::scalar(std::string s, bool quoted)
{
    Node n;
    n.kind_ = Kind::Scalar;
    n.scalar_ = std::move(s);
    n.quoted_ = quoted;
    return n;
}
Node Node::seq()
{
    Node n;
    n.kind_ = Kind::Seq;
    return n;
}
Node Node::map()
{
    Node n;
    n.kind_ = Kind::Map;
    return n;
}

size_t Node::size() const
{
    if (kind_ == Kind::Seq) return items_.size();
    if (kind_ == Kind::Map) return entries_.size();
    return 0;
}

const Node& Node::operator[](size_t i) const
{
    if (kind_ != Kind::Seq || i >= items_.size()) return nullNode();
    return items_[i];
}

const Node& Node::operator[](const std::string& key) const
{
    if (kind_ != Kind::Map) return nullNode();
    for (const auto& kv : entries_)
        if (kv.first.isScalar() && kv.first.scalar_ == key) return kv.second;
    return nullNode();
}

const std::string& Node::str() const
{
    if (kind_ != Kind::Scalar) throw ParseError("yaml: expected a scalar");
    return scalar_;
}

double Node::asDouble() const
{
    const std::string& s = str();
    if (s.empty()) throw ParseError("yaml: empty scalar where a number is expected");
    const char* b = s.c_str();
    char* e = nullptr;
    errno = 0;
    double v = std::strtod(b, &e);
    while (e && *e && std::isspace((unsigned char)*e)) ++e;
    if (e == b || (e && *e)) throw ParseError("yaml: bad number '" + s + "'");
    return v;
}

int Node::asInt() const
{
    double v = asDouble();
    int iv = (int)v;
    if ((double)iv != v) throw ParseError("yaml: bad integer '" + str() + "'");
    return iv;
}

bool Node::asBool() const
{
    std::string s = str();
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    if (s == "true" || s == "yes" || s == "y" || s == "on" || s == "1") return true;
    if (s == "false" || s == "no" || s == "n" || s == "off" || s == "0") return false;
    throw ParseError("yaml: bad boolean '" + str() + "'");
}

std::vector<std::string> Node::asStrings() const
{
    if (kind_ != Kind::Seq) throw ParseError("yaml: expected a sequence of strings");
    std::vector<std::string> out;
    for (const auto& it : items_) out.push_back(it.str());
    return out;
}

std::vector<double> Node::asDoubles() const
{
    if (kind_ != Kind::Seq) throw ParseError("yaml: expected a sequence of numbers");
    std::vector<double> out;
    for (const auto& it : items_) out.push_back(it.asDouble());
    return out;
}

std::vector<int> Node::asInts() const
{
    if (kind_ != Kind::Seq) throw ParseError("yaml: expected a sequence of integers");
    std::vector<int> out;
    for (const auto& it : items_) out.push_back(it.asInt());
    return out;
}

// ---------------------------------------------------------------------------
// Parser
// ---------------------------------------------------------------------------
namespace {

struct Line {
    int indent;
    std::string text;  // comment-stripped, right-trimmed, indentation removed
    int lineno;
};

std::string rtrim(const std::string& s)
{
    size_t e = s.find_last_not_of(" \t\r\n");
    return e == std::string::npos ? std::string() : s.substr(0, e + 1);
}
std::string trim(const std::string& s)
{
    size_t b = s.find_first_not_of(" \t\r\n");
    if (b == std::string::npos) return std::string();
    size_t e = s.find_last_not_of(" \t\r\n");
    return s.substr(b, e - b + 1);
}

// Remove a trailing comment: '#' at the start or after whitespace, outside quotes.
std::string stripComment(const std::string& s)
{
    bool sq = false, dq = false;
    for (size_t i = 0; i < s.size(); ++i) {
        char c = s[i];
        if (dq) {
            if (c == '\\') { ++i; continue; }
            if (c == '"') dq = false;
            continue;
        }
        if (sq) {
            if (c == '\'') {
                if (i + 1 < s.size() && s[i + 1] == '\'') { ++i; continue; }
                sq = false;
            }
            continue;
        }
        if (c == '"') { dq = true; continue; }
        if (c == '\'') { sq = true; continue; }
        if (c == '#' && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t')) return s.substr(0, i);
    }
    return s;
}

bool isSeqItem(const std::string& t)
{
    return !t.empty() && t[0] == '-' && (t.size() == 1 || t[1] == ' ' || t[1] == '\t');
}

// Position of the top-level mapping ':' (followed by blank or end), or npos.
size_t findMapColon(const std::string& t)
{
    int depth = 0;
    bool sq = false, dq = false;
    for (size_t i = 0; i < t.size(); ++i) {
        char c = t[i];
        if (dq) {
            if (c == '\\') { ++i; continue; }
            if (c == '"') dq = false;
            continue;
        }
        if (sq) {
            if (c == '\'') {
                if (i + 1 < t.size() && t[i + 1] == '\'') { ++i; continue; }
                sq = false;
            }
            continue;
        }
        if (c == '"' && (i == 0 || depth > 0 || t[i - 1] == ' ' || t[i - 1] == '[' || t[i - 1] == '{' || t[i - 1] == ',')) { dq = true; continue; }
        if (c == '\'' && (i == 0 || depth > 0 || t[i - 1] == ' ' || t[i - 1] == '[' || t[i - 1] == '{' || t[i - 1] == ',')) { sq = true; continue; }
        if (c == '[' || c == '{') { ++depth; continue; }
        if (c == ']' || c == '}') { if (depth > 0) --depth; continue; }
        if (c == ':' && depth == 0 && (i + 1 == t.size() || t[i + 1] == ' ' || t[i + 1] == '\t'))
            return i;
    }
    return std::string::npos;
}

int bracketBalance(const std::string& t)
{
    int depth = 0;
    bool sq = false, dq = false;
    for (size_t i = 0; i < t.size(); ++i) {
        char c = t[i];
        if (dq) {
            if (c == '\\') { ++i; continue; }
            if (c == '"') dq = false;
            continue;
        }
        if (sq) {
            if (c == '\'') {
                if (i + 1 < t.size() && t[i + 1] == '\'') { ++i; continue; }
                sq = false;
            }
            continue;
        }
        if (c == '"') dq = true;
        else if (c == '\'') sq = true;
        else if (c == '[' || c == '{') ++depth;
        else if (c == ']' || c == '}') --depth;
    }
    return depth;
}

class Parser {
public:
    explicit Parser(const std::string& text)
    {
        std::istringstream in(text);
        std::string raw;
        int ln = 0;
        while (std::getline(in, raw)) {
            ++ln;
            std::string s = rtrim(stripComment(raw));
            if (trim(s).empty()) continue;
            size_t ind = s.find_first_not_of(' ');
            if (s[ind] == '\t') throw err(ln, "tab indentation is not allowed");
            std::string t = s.substr(ind);
            if (ind == 0 && (t == "---" || t == "...")) continue;
            lines_.push_back({(int)ind, t, ln});
        }
    }

    Node parseDocument()
    {
        if (lines_.empty()) return Node();
        Node n = parseBlock(lines_[0].indent);
        if (pos_ < lines_.size()) throw err(lines_[pos_].lineno, "unexpected content: " + lines_[pos_].text);
        return n;
    }

private:
    std::vector<Line> lines_;
    size_t pos_ = 0;

    static ParseError err(int ln, const std::string& m)
    {
        return ParseError("yaml line " + std::to_string(ln) + ": " + m);
    }

    Node parseBlock(int indent)
    {
        if (pos_ >= lines_.size()) return Node();
        if (isSeqItem(lines_[pos_].text)) return parseSeq(indent);
        if (findMapColon(lines_[pos_].text) != std::string::npos) return parseMap(indent);
        // A lone scalar / flow node at block level.
        std::string t = lines_[pos_].text;
        int ln = lines_[pos_].lineno;
        ++pos_;
        return parseInline(t, ln, indent);
    }

    Node parseSeq(int indent)
    {
        Node seq = Node::seq();
        while (pos_ < lines_.size() && lines_[pos_].indent == indent && isSeqItem(lines_[pos_].text)) {
            Line& L = lines_[pos_];
            std::string rest = L.text.substr(1);
            size_t sp = rest.find_first_not_of(" \t");
            if (sp == std::string::npos) {
                ++pos_;
                if (pos_ < lines_.size() && lines_[pos_].indent > indent)
                    seq.push(parseBlock(lines_[pos_].indent));
                else
                    seq.push(Node());
                continue;
            }
            int col = indent + 1 + (int)sp;
            rest = rest.substr(sp);
            if (isSeqItem(rest) || findMapColon(rest) != std::string::npos) {
                // Re-interpret the remainder of this line as a nested block at its column.
                L.indent = col;
                L.text = rest;
                seq.push(parseBlock(col));
            } else {
                int ln = L.lineno;
                ++pos_;
                seq.push(parseInline(rest, ln, indent));
            }
        }
        return seq;
    }

    Node parseMap(int indent)
    {
        Node map = Node::map();
        while (pos_ < lines_.size() && lines_[pos_].indent == indent && !isSeqItem(lines_[pos_].text)) {
            const Line L = lines_[pos_];
            size_t c = findMapColon(L.text);
            if (c == std::string::npos) throw err(L.lineno, "expected 'key: value', got: " + L.text);
            std::string kt = trim(L.text.substr(0, c));
            std::string vt = trim(L.text.substr(c + 1));
            Node key = parseFlowText(kt, L.lineno);
            ++pos_;
            Node val;
            if (vt.empty()) {
                if (pos_ < lines_.size() && lines_[pos_].indent > indent)
                    val = parseBlock(lines_[pos_].indent);
                else if (pos_ < lines_.size() && lines_[pos_].indent == indent && isSeqItem(lines_[pos_].text))
                    val = parseSeq(indent);
            } else {
                val = parseInline(vt, L.lineno, indent);
            }
            map.add(std::move(key), std::move(val));
        }
        return map;
    }

    // A value given on the same line as its key / dash. Flow collections may
    // continue on following lines; '|' and '>' block scalars are collected.
    Node parseInline(std::string t, int ln, int parentIndent)
    {
        if (t == "|" || t == ">" || t == "|-" || t == ">-") {
            bool literal = t[0] == '|';
            std::string acc;
            while (pos_ < lines_.size() && lines_[pos_].indent > parentIndent) {
                if (!acc.empty()) acc += literal ? "\n" : " ";
                acc += lines_[pos_].text;
                ++pos_;
            }
            return Node::scalar(acc, true);
        }
        if (!t.empty() && (t[0] == '[' || t[0] == '{')) {
            while (bracketBalance(t) > 0 && pos_ < lines_.size()) {
                t += " " + lines_[pos_].text;
                ++pos_;
            }
        }
        return parseFlowText(t, ln);
    }

    Node parseFlowText(const std::string& t, int ln)
    {
        size_t p = 0;
        Node n = parseFlowNode(t, p, ln, false);
        skipSpaces(t, p);
        if (p != t.size()) {
            // Plain block scalars may legally contain flow indicators; keep the
            // full text as a scalar (yaml-cpp behaves the same for e.g. "a, b").
            // Flow collections followed by more text (seen in Plot sections,
            // e.g. "bins: [100, 100]; range: [...]") are kept as one scalar too.
            (void)ln;
            return Node::scalar(trim(t));
        }
        return n;
    }

    static void skipSpaces(const std::string& t, size_t& p)
    {
        while (p < t.size() && (t[p] == ' ' || t[p] == '\t')) ++p;
    }

    Node parseFlowNode(const std::string& t, size_t& p, int ln, bool inFlow)
    {
        skipSpaces(t, p);
        if (p >= t.size()) return Node();
        char c = t[p];
        if (c == '[') {
            ++p;
            Node seq = Node::seq();
            while (true) {
                skipSpaces(t, p);
                if (p >= t.size()) throw err(ln, "unterminated '['");
                if (t[p] == ']') { ++p; break; }
                Node elem = parseFlowNode(t, p, ln, true);
                skipSpaces(t, p);
                if (p < t.size() && t[p] == ':' && (p + 1 == t.size() || t[p + 1] == ' ' || t[p + 1] == ',' || t[p + 1] == ']')) {
                    // single-pair mapping inside a flow sequence
                    ++p;
                    skipSpaces(t, p);
                    Node val;
                    if (p < t.size() && t[p] != ',' && t[p] != ']') val = parseFlowNode(t, p, ln, true);
                    Node m = Node::map();
                    m.add(std::move(elem), std::move(val));
                    elem = std::move(m);
                    skipSpaces(t, p);
                }
                seq.push(std::move(elem));
                if (p < t.size() && t[p] == ',') { ++p; continue; }
                if (p < t.size() && t[p] == ']') { ++p; break; }
                throw err(ln, "expected ',' or ']' in flow sequence");
            }
            return seq;
        }
        if (c == '{') {
            ++p;
            Node map = Node::map();
            while (true) {
                skipSpaces(t, p);
                if (p >= t.size()) throw err(ln, "unterminated '{'");
                if (t[p] == '}') { ++p; break; }
                Node key = parseFlowNode(t, p, ln, true);
                skipSpaces(t, p);
                Node val;
                if (p < t.size() && t[p] == ':') {
                    ++p;
                    skipSpaces(t, p);
                    if (p < t.size() && t[p] != ',' && t[p] != '}') val = parseFlowNode(t, p, ln, true);
                }
                map.add(std::move(key), std::move(val));
                skipSpaces(t, p);
                if (p < t.size() && t[p] == ',') { ++p; continue; }
                if (p < t.size() && t[p] == '}') { ++p; break; }
                throw err(ln, "expected ',' or '}' in flow mapping");
            }
            return map;
        }
        if (c == '"') {
            ++p;
            std::string s;
            while (p < t.size() && t[p] != '"') {
                if (t[p] == '\\' && p + 1 < t.size()) {
                    char e = t[p + 1];
                    switch (e) {
                    case 'n': s += '\n'; break;
                    case 't': s += '\t'; break;
                    case 'r': s += '\r'; break;
                    case '0': s += '\0'; break;
                    default: s += e; break;
                    }
                    p += 2;
                } else {
                    s += t[p++];
                }
            }
            if (p >= t.size()) throw err(ln, "unterminated double-quoted scalar");
            ++p;
            return Node::scalar(s, true);
        }
        if (c == '\'') {
            ++p;
            std::string s;
            while (p < t.size()) {
                if (t[p] == '\'') {
                    if (p + 1 < t.size() && t[p + 1] == '\'') { s += '\''; p += 2; continue; }
                    break;
                }
                s += t[p++];
            }
            if (p >= t.size()) throw err(ln, "unterminated single-quoted scalar");
            ++p;
            return Node::scalar(s, true);
        }
        // Plain scalar.
        size_t b = p;
        while (p < t.size()) {
            char d = t[p];
            if (inFlow && (d == ',' || d == ']' || d == '}')) break;
            if (d == ':' && (p + 1 == t.size() || t[p + 1] == ' ' || (inFlow && (t[p + 1] == ',' || t[p + 1] == ']' || t[p + 1] == '}')))) break;
            ++p;
        }
        std::string s = trim(t.substr(b, p - b));
        if (s.empty() || s == "~" || s == "null" || s == "Null" || s == "NULL") return Node();
        return Node::scalar(s);
    }
};

}  // namespace

Node parse(const std::string& text)
{
    Parser p(text);
    return p.parseDocument();
}

Node parseFile(const std::string& path)
{
    std::ifstream f(path);
    if (!f.is_open()) throw ParseError("yaml: cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return parse(ss.str());
}

}  // namespace yaml
}  // namespace ctpwa
