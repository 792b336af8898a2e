// dot.hh -- a small GraphViz DOT reader for roadmap graphs, replacing the
// reference driver's Boost read_graphviz call (scripts/batch_cc.cpp:281-328).
//
// Reads `graph` / `digraph` files whose vertices carry a `states` attribute
// (whitespace-separated joint values) and returns the edges in file order, each
// as its two endpoint state vectors, source first.  Vertices are identified by
// their DOT ids (the reference reads with "node_id"); attributes other than
// `states` are ignored, as the reference's ignore_other_properties does.
// Supported statements: node statements, edge statements (chains a -- b -- c
// included), attribute statements (graph/node/edge [...]) and `id = id`
// assignments; subgraphs are rejected with an error.
#pragma once

#include <cctype>
#include <cstring>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace bcc_dot {

struct Graph {
    std::vector<std::vector<double>> states;  // per vertex, in order of first appearance
    std::vector<std::pair<int, int>> edges;   // (source, target) vertex indices, file order
};

class Lexer {
   public:
    explicit Lexer(const std::string& s) : s_(s) {}

    // Next token: an id / number / quoted string (quotes removed, kind 'i'), or a
    // punctuation token ('{', '}', '[', ']', '=', ';', ',', and "--" / "->" as 'e').
    bool next(std::string& tok, char& kind) {
        skip();
        if (i_ >= s_.size()) return false;
        const char c = s_[i_];
        if (c == '"') {
            std::string out;
            for (++i_; i_ < s_.size() && s_[i_] != '"'; ++i_) {
                if (s_[i_] == '\\' && i_ + 1 < s_.size()) ++i_;
                out += s_[i_];
            }
            if (i_ >= s_.size()) throw std::runtime_error("DOT: unterminated string");
            ++i_;
            tok = out;
            kind = 'i';
            return true;
        }
        if (c == '-' && i_ + 1 < s_.size() && (s_[i_ + 1] == '-' || s_[i_ + 1] == '>')) {
            tok = s_.substr(i_, 2);
            i_ += 2;
            kind = 'e';
            return true;
        }
        if (c != '\0' && std::strchr("{}[]=;,", c)) {
            tok = std::string(1, c);
            ++i_;
            kind = c;
            return true;
        }
        std::string out;
        while (i_ < s_.size() && (std::isalnum((unsigned char)s_[i_]) || s_[i_] == '_' || s_[i_] == '.' ||
                                  (s_[i_] == '-' && !(i_ + 1 < s_.size() && (s_[i_ + 1] == '-' || s_[i_ + 1] == '>')))))
            out += s_[i_++];
        if (out.empty()) throw std::runtime_error(std::string("DOT: unexpected character '") + c + "'");
        tok = out;
        kind = 'i';
        return true;
    }

   private:
    void skip() {
        for (;;) {
            while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_;
            if (s_.compare(i_, 2, "//") == 0 || (i_ < s_.size() && s_[i_] == '#')) {
                while (i_ < s_.size() && s_[i_] != '\n') ++i_;
            } else if (s_.compare(i_, 2, "/*") == 0) {
                const size_t e = s_.find("*/", i_ + 2);
                i_ = e == std::string::npos ? s_.size() : e + 2;
            } else {
                return;
            }
        }
    }
    const std::string& s_;
    size_t i_ = 0;
};

inline Graph parse(const std::string& text) {
    Lexer lx(text);
    std::string tok;
    char kind;
    Graph g;
    std::map<std::string, int> id;
    auto vertex = [&](const std::string& name) {
        auto it = id.find(name);
        if (it != id.end()) return it->second;
        const int v = (int)g.states.size();
        id[name] = v;
        g.states.emplace_back();
        return v;
    };
    // header: [strict] (graph|digraph) [id] {
    if (!lx.next(tok, kind)) throw std::runtime_error("DOT: empty file");
    if (tok == "strict" && !lx.next(tok, kind)) throw std::runtime_error("DOT: truncated header");
    if (tok != "graph" && tok != "digraph") throw std::runtime_error("DOT: expected graph or digraph");
    if (!lx.next(tok, kind)) throw std::runtime_error("DOT: truncated header");
    if (kind == 'i' && !lx.next(tok, kind)) throw std::runtime_error("DOT: truncated header");
    if (kind != '{') throw std::runtime_error("DOT: expected '{'");

    // [a=b, c=d] -> the value of `states`, if any
    auto attr_list = [&](std::string* states) {
        for (;;) {
            if (!lx.next(tok, kind)) throw std::runtime_error("DOT: unterminated attribute list");
            if (kind == ']') return;
            if (kind == ',' || kind == ';') continue;
            if (kind != 'i') throw std::runtime_error("DOT: bad attribute list");
            const std::string key = tok;
            if (!lx.next(tok, kind) || kind != '=') throw std::runtime_error("DOT: expected '=' in attribute list");
            if (!lx.next(tok, kind) || kind != 'i') throw std::runtime_error("DOT: expected attribute value");
            if (states && key == "states") *states = tok;
        }
    };

    bool have = lx.next(tok, kind);
    while (have) {
        if (kind == '}') return g;
        if (kind == ';' || kind == ',') {
            have = lx.next(tok, kind);
            continue;
        }
        if (kind != 'i') throw std::runtime_error("DOT: unexpected '" + tok + "'");
        if (tok == "subgraph") throw std::runtime_error("DOT: subgraphs are not supported");
        if (tok == "graph" || tok == "node" || tok == "edge") {  // default attributes
            if (lx.next(tok, kind) && kind == '[') attr_list(nullptr);
            have = lx.next(tok, kind);
            continue;
        }
        std::string first = tok;
        have = lx.next(tok, kind);
        if (have && kind == '=') {  // graph attribute id = id
            lx.next(tok, kind);
            have = lx.next(tok, kind);
            continue;
        }
        std::vector<int> chain{vertex(first)};
        while (have && kind == 'e') {
            if (!lx.next(tok, kind) || kind != 'i') throw std::runtime_error("DOT: expected a vertex after an edge op");
            chain.push_back(vertex(tok));
            have = lx.next(tok, kind);
        }
        std::string states;
        if (have && kind == '[') {
            attr_list(chain.size() == 1 ? &states : nullptr);
            have = lx.next(tok, kind);
        }
        if (chain.size() == 1) {
            if (!states.empty()) {
                std::istringstream in(states);
                std::vector<double> v;
                double x;
                while (in >> x) v.push_back(x);
                g.states[chain[0]] = v;
            }
        } else {
            for (size_t k = 0; k + 1 < chain.size(); ++k) g.edges.emplace_back(chain[k], chain[k + 1]);
        }
    }
    throw std::runtime_error("DOT: missing '}'");
}

}  // namespace bcc_dot
