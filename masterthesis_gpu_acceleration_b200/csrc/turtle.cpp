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

#include <cctype>
#include <cstdio>
#include <fstream>
#include <sstream>

namespace gr {
namespace {

inline bool is_space(char c) { return std::isspace((unsigned char)c) != 0; }
inline bool is_name_char(char c) {
    unsigned char u = (unsigned char)c;
    return std::isalnum(u) || c == '_' || c == '-' || c == '.' || u >= 128;
}

class Reader {
public:
    Reader(const std::string& s, TermDict& e, TermDict& p, std::vector<int32_t>& out)
        : src_(s), ents_(e), preds_(p), out_(out) {}

    void run() {
        for (;;) {
            skip_ws();
            if (pos_ >= src_.size()) break;
            if (src_[pos_] == '@') {
                ++pos_;
                std::string kw;
                while (pos_ < src_.size() && std::isalpha((unsigned char)src_[pos_])) kw += src_[pos_++];
                if (kw == "prefix") prefix_decl();
                else {
                    while (pos_ < src_.size() && src_[pos_] != '.') ++pos_;
                    if (pos_ < src_.size()) ++pos_;
                }
                continue;
            }
            if (sparql_prefix()) continue;
            std::string subject = term();
            if (subject.empty()) { ++pos_; continue; }
            predicate_object_list(subject);
            skip_ws();
            if (pos_ < src_.size() && src_[pos_] == '.') ++pos_;
        }
    }

private:
    const std::string& src_;
    size_t pos_ = 0;
    std::unordered_map<std::string, std::string> prefixes_;
    TermDict& ents_;
    TermDict& preds_;
    std::vector<int32_t>& out_;
    int anon_ = 0;

    void skip_ws() {
        while (pos_ < src_.size()) {
            char c = src_[pos_];
            if (is_space(c)) ++pos_;
            else if (c == '#') { while (pos_ < src_.size() && src_[pos_] != '\n') ++pos_; }
            else break;
        }
    }

    bool sparql_prefix() {
        if (src_.size() - pos_ < 6) return false;
        for (int i = 0; i < 6; ++i)
            if (std::tolower((unsigned char)src_[pos_ + i]) != "prefix"[i]) return false;
        if (src_.size() - pos_ > 6 && !is_space(src_[pos_ + 6])) return false;
        pos_ += 6;
        prefix_decl();
        return true;
    }

    std::string iri() {
        ++pos_;
        size_t b = pos_;
        while (pos_ < src_.size() && src_[pos_] != '>') ++pos_;
        std::string s = src_.substr(b, pos_ - b);
        if (pos_ < src_.size()) ++pos_;
        return s;
    }

    // Reads name characters, then gives trailing dots back to the input.
    std::string name_run() {
        size_t b = pos_;
        while (pos_ < src_.size() && is_name_char(src_[pos_])) ++pos_;
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
        bool triple = pos_ + 1 < src_.size() && src_[pos_] == q && src_[pos_ + 1] == q;
        if (triple) pos_ += 2;
        std::string v;
        while (pos_ < src_.size()) {
            if (triple) {
                if (pos_ + 2 < src_.size() && src_[pos_] == q && src_[pos_ + 1] == q && src_[pos_ + 2] == q) {
                    pos_ += 3;
                    break;
                }
            } else {
                if (src_[pos_] == q) { ++pos_; break; }
                if (src_[pos_] == '\n') break;
            }
            if (src_[pos_] == '\\' && pos_ + 1 < src_.size()) {
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
        if (pos_ >= src_.size()) return "";
        char c = src_[pos_];
        if (c == '<') return iri();
        if (c == '_' && pos_ + 1 < src_.size() && src_[pos_ + 1] == ':') {
            pos_ += 2;
            size_t b = pos_;
            while (pos_ < src_.size()) {
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
            if (pos_ < src_.size() && src_[pos_] == ']') ++pos_;
            return "_:anon" + std::to_string(++anon_);
        }
        if (c == '"' || c == '\'') {
            std::string lit = "\"" + quoted() + "\"";
            skip_ws();
            if (pos_ < src_.size() && src_[pos_] == '@') {
                ++pos_;
                std::string lang;
                while (pos_ < src_.size() && (std::isalnum((unsigned char)src_[pos_]) || src_[pos_] == '-'))
                    lang += src_[pos_++];
                lit += "@" + lang;
            } else if (pos_ + 1 < src_.size() && src_[pos_] == '^' && src_[pos_ + 1] == '^') {
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
            if (pos_ < src_.size() && src_[pos_] == ':') return expand(ident);
            if (ident == "a") return "http://www.w3.org/1999/02/22-rdf-syntax-ns#type";
            if (ident == "true") return "\"true\"^^http://www.w3.org/2001/XMLSchema#boolean";
            if (ident == "false") return "\"false\"^^http://www.w3.org/2001/XMLSchema#boolean";
            return ident;
        }
        if (std::isdigit((unsigned char)c) || c == '+' || c == '-') {
            size_t b = pos_;
            while (pos_ < src_.size()) {
                char ch = src_[pos_];
                if (std::isdigit((unsigned char)ch) || ch == '.' || ch == 'e' || ch == 'E' || ch == '+' || ch == '-') ++pos_;
                else break;
            }
            return "\"" + src_.substr(b, pos_ - b) + "\"";
        }
        return "";
    }

    void prefix_decl() {
        skip_ws();
        std::string name;
        while (pos_ < src_.size() && src_[pos_] != ':') {
            if (!is_space(src_[pos_])) name += src_[pos_];
            ++pos_;
        }
        if (pos_ < src_.size()) ++pos_;
        skip_ws();
        std::string uri;
        if (pos_ < src_.size() && src_[pos_] == '<') uri = iri();
        prefixes_[name] = uri;
        skip_ws();
        if (pos_ < src_.size() && src_[pos_] == '.') ++pos_;
    }

    void emit(const std::string& s, const std::string& p, const std::string& o) {
        out_.push_back(ents_.intern(s));
        out_.push_back(preds_.intern(p));
        out_.push_back(ents_.intern(o));
    }

    void predicate_object_list(const std::string& subject) {
        for (;;) {
            skip_ws();
            if (pos_ >= src_.size() || src_[pos_] == '.' || src_[pos_] == ']') break;
            if (src_[pos_] == ';') {
                ++pos_;
                skip_ws();
                if (pos_ < src_.size() && (src_[pos_] == '.' || src_[pos_] == ']')) break;
                continue;
            }
            std::string pred = term();
            if (pred.empty()) break;
            for (;;) {
                std::string obj = term();
                if (!obj.empty()) emit(subject, pred, obj);
                skip_ws();
                if (pos_ < src_.size() && src_[pos_] == ',') { ++pos_; continue; }
                break;
            }
            skip_ws();
            if (pos_ < src_.size() && src_[pos_] == ';') { ++pos_; continue; }
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

bool parse_turtle_file(const std::string& path, TermDict& ents, TermDict& preds,
                       std::vector<int32_t>& spo, std::string* err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        if (err) *err = "cannot open " + path;
        return false;
    }
    std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    return parse_turtle_text(text, ents, preds, spo);
}

std::unordered_map<std::string, std::string> scan_rule_prefixes(const std::string& path) {
    std::unordered_map<std::string, std::string> out;
    std::ifstream in(path);
    if (!in) return out;
    std::string line;
    while (std::getline(in, line)) {
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
