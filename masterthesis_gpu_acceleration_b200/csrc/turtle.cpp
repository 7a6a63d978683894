// turtle.cpp — Turtle reader accepting the reference's syntax subset.
//
// Term spellings follow the reference's reader so that rule constants
// resolve to the same terms (CPU_01_nonparallel/RdfIndexes.cpp:168-309):
//   <iri>           -> iri (brackets dropped, no escape processing)
//   pfx:local       -> expansion of pfx + local, or "pfx:local" if unknown
//   :local          -> default-prefix expansion, or ":local"
//   _:label, []     -> "_:label", "_:anonN"
//   "text"@lang     -> "\"text\"@lang";  "text"^^T -> "\"text\"^^" + term(T)
//   a / true / false / 12.5 -> rdf:type IRI / typed booleans / "\"12.5\""
#include "turtle.hpp"

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <thread>

namespace gr {
namespace {

inline bool is_space(char c) { return std::isspace((unsigned char)c) != 0; }
inline bool is_name_char(char c) {
    unsigned char u = (unsigned char)c;
    return std::isalnum(u) || c == '_' || c == '-' || c == '.' || u >= 128;
}

class Reader {
public:
    Reader(const std::string& s, TermDict& e, TermDict& p, std::vector<int32_t>& out, size_t begin = 0,
           size_t end = std::string::npos)
        : src_(s), end_(std::min(end, s.size())), pos_(begin), ents_(e), preds_(p), out_(out) {}

    const std::unordered_map<std::string, std::string>& prefixes() const { return prefixes_; }
    bool saw_prefix() const { return sawPrefix_; }
    void set_prefixes(const std::unordered_map<std::string, std::string>& p) { prefixes_ = p; }

    void run() {
        for (;;) {
            skip_ws();
            if (pos_ >= end_) break;
            if (src_[pos_] == '@') {
                ++pos_;
                std::string kw;
                while (pos_ < end_ && std::isalpha((unsigned char)src_[pos_])) kw += src_[pos_++];
                if (kw == "prefix") prefix_decl();
                else {
                    while (pos_ < end_ && src_[pos_] != '.') ++pos_;
                    if (pos_ < end_) ++pos_;
                }
                continue;
            }
            if (sparql_prefix()) continue;
            std::string subject = term();
            if (subject.empty()) { ++pos_; continue; }
            predicate_object_list(subject);
            skip_ws();
            if (pos_ < end_ && src_[pos_] == '.') ++pos_;
        }
    }

private:
    const std::string& src_;
    size_t end_;      // this reader's input ends here (a chunk of the text)
    size_t pos_ = 0;
    std::unordered_map<std::string, std::string> prefixes_;
    TermDict& ents_;
    TermDict& preds_;
    std::vector<int32_t>& out_;
    int anon_ = 0;
    bool sawPrefix_ = false;

    void skip_ws() {
        while (pos_ < end_) {
            char c = src_[pos_];
            if (is_space(c)) ++pos_;
            else if (c == '#') { while (pos_ < end_ && src_[pos_] != '\n') ++pos_; }
            else break;
        }
    }

    bool sparql_prefix() {
        if (end_ - pos_ < 6) return false;
        for (int i = 0; i < 6; ++i)
            if (std::tolower((unsigned char)src_[pos_ + i]) != "prefix"[i]) return false;
        if (end_ - pos_ > 6 && !is_space(src_[pos_ + 6])) return false;
        pos_ += 6;
        prefix_decl();
        return true;
    }

    std::string iri() {
        ++pos_;
        size_t b = pos_;
        while (pos_ < end_ && src_[pos_] != '>') ++pos_;
        std::string s = src_.substr(b, pos_ - b);
        if (pos_ < end_) ++pos_;
        return s;
    }

    // Reads name characters, then gives trailing dots back to the input.
    std::string name_run() {
        size_t b = pos_;
        while (pos_ < end_ && is_name_char(src_[pos_])) ++pos_;
        while (pos_ > b && src_[pos_ - 1] == '.') --pos_;
        return src_.substr(b, pos_ - b);
    }

    std::string expand(const std::string& pfx) {
        ++pos_;  // ':'
        std::string local = name_run();
        auto it = prefixes_.find(pfx);
        return it != prefixes_.end() ? it->second + local : pfx + ":" + local;
    }

    std::string quoted() {
        char q = src_[pos_++];
        bool triple = pos_ + 1 < end_ && src_[pos_] == q && src_[pos_ + 1] == q;
        if (triple) pos_ += 2;
        std::string v;
        while (pos_ < end_) {
            if (triple) {
                if (pos_ + 2 < end_ && src_[pos_] == q && src_[pos_ + 1] == q && src_[pos_ + 2] == q) {
                    pos_ += 3;
                    break;
                }
            } else {
                if (src_[pos_] == q) { ++pos_; break; }
                if (src_[pos_] == '\n') break;
            }
            if (src_[pos_] == '\\' && pos_ + 1 < end_) {
                char e = src_[pos_ + 1];
                pos_ += 2;
                switch (e) {
                    case 'n': v += '\n'; break;
                    case 't': v += '\t'; break;
                    case 'r': v += '\r'; break;
                    case '\\': v += '\\'; break;
                    case '"': v += '"'; break;
                    case '\'': v += '\''; break;
                    default: v += '\\'; v += e; break;
                }
            } else {
                v += src_[pos_++];
            }
        }
        return v;
    }

    std::string term() {
        skip_ws();
        if (pos_ >= end_) return "";
        char c = src_[pos_];
        if (c == '<') return iri();
        if (c == '_' && pos_ + 1 < end_ && src_[pos_ + 1] == ':') {
            pos_ += 2;
            size_t b = pos_;
            while (pos_ < end_) {
                unsigned char u = (unsigned char)src_[pos_];
                if (std::isalnum(u) || u == '_' || u == '-' || u == '.') ++pos_;
                else break;
            }
            while (pos_ > b && src_[pos_ - 1] == '.') --pos_;
            return "_:" + src_.substr(b, pos_ - b);
        }
        if (c == '[') {
            ++pos_;
            skip_ws();
            if (pos_ < end_ && src_[pos_] == ']') ++pos_;
            return "_:anon" + std::to_string(++anon_);
        }
        if (c == '"' || c == '\'') {
            std::string lit = "\"" + quoted() + "\"";
            skip_ws();
            if (pos_ < end_ && src_[pos_] == '@') {
                ++pos_;
                std::string lang;
                while (pos_ < end_ && (std::isalnum((unsigned char)src_[pos_]) || src_[pos_] == '-'))
                    lang += src_[pos_++];
                lit += "@" + lang;
            } else if (pos_ + 1 < end_ && src_[pos_] == '^' && src_[pos_ + 1] == '^') {
                pos_ += 2;
                lit += "^^" + term();
            }
            return lit;
        }
        if (c == ':') {
            ++pos_;
            std::string local = name_run();
            auto it = prefixes_.find("");
            return it != prefixes_.end() ? it->second + local : ":" + local;
        }
        if (std::isalpha((unsigned char)c) || c == '_') {
            std::string ident = name_run();
            if (pos_ < end_ && src_[pos_] == ':') return expand(ident);
            if (ident == "a") return "http://www.w3.org/1999/02/22-rdf-syntax-ns#type";
            if (ident == "true") return "\"true\"^^http://www.w3.org/2001/XMLSchema#boolean";
            if (ident == "false") return "\"false\"^^http://www.w3.org/2001/XMLSchema#boolean";
            return ident;
        }
        if (std::isdigit((unsigned char)c) || c == '+' || c == '-') {
            size_t b = pos_;
            while (pos_ < end_) {
                char ch = src_[pos_];
                if (std::isdigit((unsigned char)ch) || ch == '.' || ch == 'e' || ch == 'E' || ch == '+' || ch == '-') ++pos_;
                else break;
            }
            return "\"" + src_.substr(b, pos_ - b) + "\"";
        }
        return "";
    }

    void prefix_decl() {
        sawPrefix_ = true;
        skip_ws();
        std::string name;
        while (pos_ < end_ && src_[pos_] != ':') {
            if (!is_space(src_[pos_])) name += src_[pos_];
            ++pos_;
        }
        if (pos_ < end_) ++pos_;
        skip_ws();
        std::string uri;
        if (pos_ < end_ && src_[pos_] == '<') uri = iri();
        prefixes_[name] = uri;
        skip_ws();
        if (pos_ < end_ && src_[pos_] == '.') ++pos_;
    }

    void emit(const std::string& s, const std::string& p, const std::string& o) {
        out_.push_back(ents_.intern(s));
        out_.push_back(preds_.intern(p));
        out_.push_back(ents_.intern(o));
    }

    void predicate_object_list(const std::string& subject) {
        for (;;) {
            skip_ws();
            if (pos_ >= end_ || src_[pos_] == '.' || src_[pos_] == ']') break;
            if (src_[pos_] == ';') {
                ++pos_;
                skip_ws();
                if (pos_ < end_ && (src_[pos_] == '.' || src_[pos_] == ']')) break;
                continue;
            }
            std::string pred = term();
            if (pred.empty()) break;
            for (;;) {
                std::string obj = term();
                if (!obj.empty()) emit(subject, pred, obj);
                skip_ws();
                if (pos_ < end_ && src_[pos_] == ',') { ++pos_; continue; }
                break;
            }
            skip_ws();
            if (pos_ < end_ && src_[pos_] == ';') { ++pos_; continue; }
            break;
        }
    }
};

}  // namespace

bool parse_turtle_text(const std::string& text, TermDict& ents, TermDict& preds, std::vector<int32_t>& spo) {
    Reader r(text, ents, preds, spo);
    r.run();
    return true;
}

namespace {

// A chunk boundary at or after `from`: just past a newline that ends a
// statement (the line's last non-space character is '.', and the line is
// not a comment).  npos if none.
size_t statement_boundary(const std::string& text, size_t from) {
    size_t nl = text.find('\n', from);
    while (nl != std::string::npos) {
        size_t b = text.rfind('\n', nl == 0 ? 0 : nl - 1);
        b = (b == std::string::npos || b >= nl) ? 0 : b + 1;
        size_t e = nl;
        while (e > b && is_space(text[e - 1])) --e;
        size_t f = b;
        while (f < e && is_space(text[f])) ++f;
        if (e > f && text[e - 1] == '.' && text[f] != '#') return nl + 1;
        nl = text.find('\n', nl + 1);
    }
    return std::string::npos;
}

}  // namespace

bool parse_turtle_text_parallel(const std::string& text, TermDict& ents, TermDict& preds,
                                std::vector<int32_t>& spo, size_t minChunk) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t T = std::min<size_t>(std::min(hw, 16u), text.size() / std::max<size_t>(minChunk, 1));
    // one reader when the text is small, or uses constructs whose meaning a
    // chunk cannot know (long literals that span lines, anonymous nodes
    // numbered in reading order)
    if (T < 2 || text.find("\"\"\"") != std::string::npos || text.find("'''") != std::string::npos ||
        text.find('[') != std::string::npos)
        return parse_turtle_text(text, ents, preds, spo);
    // a short first chunk holds the prefix declarations and is read first;
    // the rest is cut after statement ends and read by T threads
    std::vector<size_t> cut{0};
    const size_t head = statement_boundary(text, std::min(text.size() / T, size_t(1) << 20));
    if (head == std::string::npos || head >= text.size()) return parse_turtle_text(text, ents, preds, spo);
    cut.push_back(head);
    for (size_t k = 1; k < T; ++k) {
        const size_t b = statement_boundary(text, std::max(cut.back(), head + (text.size() - head) * k / T));
        if (b == std::string::npos || b >= text.size()) break;
        if (b > cut.back()) cut.push_back(b);
    }
    cut.push_back(text.size());
    TermDict e0, p0;
    std::vector<int32_t> s0;
    Reader first(text, e0, p0, s0, 0, cut[1]);
    first.run();
    const size_t nc = cut.size() - 1;
    std::vector<TermDict> le(nc), lp(nc);
    std::vector<std::vector<int32_t>> ls(nc);
    std::vector<char> sawPrefix(nc, 0);
    std::vector<std::thread> pool;
    for (size_t k = 1; k < nc; ++k)
        pool.emplace_back([&, k] {
            Reader r(text, le[k], lp[k], ls[k], cut[k], cut[k + 1]);
            r.set_prefixes(first.prefixes());
            r.run();
            sawPrefix[k] = r.saw_prefix() ? 1 : 0;
        });
    for (auto& th : pool) th.join();
    // a prefix declared after the first chunk changes how later chunks read:
    // read the whole text with one reader instead
    for (size_t k = 1; k < nc; ++k)
        if (sawPrefix[k]) return parse_turtle_text(text, ents, preds, spo);
    le[0] = std::move(e0);
    lp[0] = std::move(p0);
    ls[0] = std::move(s0);
    // merge in file order: global ids come out in first-seen order, as one
    // reader over the whole text assigns them
    for (size_t k = 0; k < nc; ++k) {
        std::vector<int32_t> me(le[k].size()), mp(lp[k].size());
        for (size_t i = 0; i < me.size(); ++i) me[i] = ents.intern(le[k].names[i]);
        for (size_t i = 0; i < mp.size(); ++i) mp[i] = preds.intern(lp[k].names[i]);
        const std::vector<int32_t>& v = ls[k];
        const size_t base = spo.size();
        spo.resize(base + v.size());
        for (size_t i = 0; i + 2 < v.size(); i += 3) {
            spo[base + i] = me[v[i]];
            spo[base + i + 1] = mp[v[i + 1]];
            spo[base + i + 2] = me[v[i + 2]];
        }
    }
    return true;
}

bool read_file(const std::string& path, std::string& text, std::string* err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        if (err) *err = "cannot open " + path;
        return false;
    }
    f.seekg(0, std::ios::end);
    const std::streamoff n = f.tellg();
    f.seekg(0, std::ios::beg);
    text.resize(n > 0 ? (size_t)n : 0);
    if (n > 0) f.read(&text[0], n);
    return true;
}

bool parse_turtle_file(const std::string& path, TermDict& ents, TermDict& preds,
                       std::vector<int32_t>& spo, std::string* err) {
    std::string text;
    if (!read_file(path, text, err)) return false;
    return parse_turtle_text_parallel(text, ents, preds, spo);
}

std::unordered_map<std::string, std::string> scan_rule_prefixes(const std::string& path) {
    std::string text;
    if (!read_file(path, text, nullptr)) return {};
    return scan_rule_prefixes_text(text);
}

std::unordered_map<std::string, std::string> scan_rule_prefixes_text(const std::string& text) {
    std::unordered_map<std::string, std::string> out;
    size_t pos = 0;
    while (pos < text.size()) {
        size_t nl = text.find('\n', pos);
        if (nl == std::string::npos) nl = text.size();
        // only lines whose first non-space character can start "@prefix" or
        // "prefix" are looked at (the rest of a large file is skipped fast)
        size_t f = pos;
        while (f < nl && is_space(text[f])) ++f;
        const char c0 = f < nl ? (char)std::tolower((unsigned char)text[f]) : 0;
        const size_t lineBeg = pos;
        pos = nl + 1;
        if (c0 != '@' && c0 != 'p') continue;
        std::string line = text.substr(lineBeg, nl - lineBeg);
        size_t s = 0, e = line.size();
        while (s < e && is_space(line[s])) ++s;
        while (e > s && is_space(line[e - 1])) --e;
        if (s == e) continue;
        std::string t = line.substr(s, e - s);
        std::string low = t;
        for (auto& c : low) c = (char)std::tolower((unsigned char)c);
        size_t nameStart;
        if (low.compare(0, 7, "@prefix") == 0) nameStart = 7;
        else if (low.compare(0, 6, "prefix") == 0) nameStart = 6;
        else continue;
        while (nameStart < t.size() && is_space(t[nameStart])) ++nameStart;
        size_t colon = t.find(':', nameStart);
        if (colon == std::string::npos) continue;
        std::string name = t.substr(nameStart, colon - nameStart);
        size_t ns = 0, ne = name.size();
        while (ns < ne && is_space(name[ns])) ++ns;
        while (ne > ns && is_space(name[ne - 1])) --ne;
        name = name.substr(ns, ne - ns);
        size_t ub = t.find('<', colon);
        if (ub == std::string::npos) continue;
        size_t ue = t.find('>', ub);
        if (ue == std::string::npos) continue;
        std::string uri = t.substr(ub + 1, ue - ub - 1);
        if (!name.empty() && !uri.empty()) out[name] = uri;
    }
    return out;
}

}  // namespace gr
