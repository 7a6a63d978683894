// rules.cpp — rule text / JSON front-end with the reference's accepted syntax.
#include "rules.hpp"

#include <cctype>

namespace gr {
namespace {

std::string_view trim(std::string_view s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
}

// The first three whitespace-separated tokens of s, as
// `istringstream(s) >> a >> b >> c` reads them (RuleParser.cpp reads an atom
// that way): leading whitespace skipped, missing tokens left empty, anything
// after the third ignored.
void three_tokens(std::string_view s, std::string_view& a, std::string_view& b, std::string_view& c) {
    std::string_view* out[3] = {&a, &b, &c};
    size_t i = 0;
    const size_t n = s.size();
    for (std::string_view* t : out) {
        while (i < n && std::isspace((unsigned char)s[i])) ++i;
        size_t j = i;
        while (j < n && !std::isspace((unsigned char)s[j])) ++j;
        *t = s.substr(i, j - i);
        i = j;
    }
}

// Calls fn(atom) for the body's atoms: split on '^' outside parentheses,
// trimmed, empty ones skipped (RuleParser.cpp:155-184).
template <class Fn>
void for_atoms(std::string_view body, Fn fn) {
    int depth = 0;
    size_t start = 0;
    for (size_t i = 0; i < body.size(); ++i) {
        const char ch = body[i];
        if (ch == '(') ++depth;
        else if (ch == ')') --depth;
        else if (ch == '^' && depth == 0) {
            const std::string_view t = trim(body.substr(start, i - start));
            if (!t.empty()) fn(t);
            start = i + 1;
        }
    }
    const std::string_view t = trim(body.substr(start));
    if (!t.empty()) fn(t);
}

// "key": "value" lookup without escape handling (RuleParser.cpp:10-21).
std::string json_str(const std::string& obj, const std::string& key) {
    std::string k = "\"" + key + "\"";
    size_t p = obj.find(k);
    if (p == std::string::npos) return "";
    p += k.size();
    while (p < obj.size() && (obj[p] == ' ' || obj[p] == '\t' || obj[p] == ':' || obj[p] == '\n' || obj[p] == '\r')) ++p;
    if (p >= obj.size() || obj[p] != '"') return "";
    ++p;
    size_t e = obj.find('"', p);
    if (e == std::string::npos) return "";
    return obj.substr(p, e - p);
}

// Brace-matched object starting at `start` (RuleParser.cpp:23-30).
std::string json_object_at(const std::string& s, size_t start) {
    int depth = 0;
    for (size_t i = start; i < s.size(); ++i) {
        if (s[i] == '{') ++depth;
        else if (s[i] == '}') {
            if (--depth == 0) return s.substr(start, i - start + 1);
        }
    }
    return "";
}

std::vector<std::string> json_objects(const std::string& arr) {
    std::vector<std::string> out;
    for (size_t i = 0; i < arr.size(); ++i) {
        if (arr[i] == '{') {
            std::string o = json_object_at(arr, i);
            if (!o.empty()) { out.push_back(o); i += o.size() - 1; }
        }
    }
    return out;
}

}  // namespace

void RuleParser::expand(std::string_view token, std::string& out) const {
    if (token.size() >= 2 && token.front() == '<' && token.back() == '>') {
        out.assign(token.substr(1, token.size() - 2));
        return;
    }
    if (!token.empty() && token.front() != '?' && token.front() != '"') {
        const size_t c = token.find(':');
        if (c != std::string_view::npos) {
            out.assign(token.substr(0, c));
            auto it = prefixes_.find(out);
            if (it != prefixes_.end()) {
                out = it->second;
                out.append(token.substr(c + 1));
                return;
            }
        }
    }
    out.assign(token);
}

Term RuleParser::var_term(std::string_view name, Scope& sc) const {
    Term t;
    t.isVar = true;
    for (const auto& v : sc.vars)
        if (std::string_view(v.first) == name) { t.id = v.second; return t; }
    t.id = sc.nextVar++;
    sc.vars.emplace_back(std::string(name), t.id);
    return t;
}

Term RuleParser::const_term(const std::string& spelled, Scope& sc) const {
    Term t;
    t.isVar = false;
    int32_t id = ents_.find(spelled);
    if (id >= 0) { t.id = id; return t; }
    for (const auto& u : sc.unknown)
        if (u.first == spelled) { t.id = u.second; return t; }
    t.id = -1 - (int32_t)sc.unknown.size();
    sc.unknown.emplace_back(spelled, t.id);
    return t;
}

Term RuleParser::text_term(std::string_view token, Scope& sc) const {
    const std::string_view c = trim(token);
    if (c.empty()) throw RuleError("Empty term token");
    if (c.front() == '?') return var_term(c, sc);
    static thread_local std::string key;   // reused: no allocation per term once grown
    expand(c, key);
    return const_term(key, sc);
}

int32_t RuleParser::pred_id(std::string_view token) const {
    static thread_local std::string key;
    expand(token, key);
    return preds_.find(key);
}

Rule RuleParser::parse_text(const std::string& line) const {
    std::string_view clean = trim(line);
    if (clean.empty()) throw RuleError("Empty rule line");
    const size_t bar = clean.find('|');
    if (bar != std::string_view::npos) clean = trim(clean.substr(0, bar));
    const size_t arrow = clean.find("=>");
    if (arrow == std::string_view::npos) throw RuleError("Rule line missing => : " + line);
    const std::string_view bodyText = trim(clean.substr(0, arrow));
    const std::string_view headText = trim(clean.substr(arrow + 2));
    Scope sc;
    Rule r;
    auto atom_of = [&](std::string_view raw, const char* what) {
        const std::string_view s = trim(raw);
        if (s.empty() || s.front() != '(' || s.back() != ')')
            throw RuleError(std::string("Invalid ") + what + ": " + std::string(raw));
        std::string_view st, pt, ot;
        three_tokens(s.substr(1, s.size() - 2), st, pt, ot);
        if (st.empty() || pt.empty() || ot.empty())
            throw RuleError(std::string("Invalid ") + what + ": " + std::string(raw));
        Atom a;
        a.s = text_term(st, sc);
        a.o = text_term(ot, sc);
        a.pred = pred_id(pt);
        return a;
    };
    for_atoms(bodyText, [&](std::string_view a) { r.body.push_back(atom_of(a, "body atom")); });
    r.head = atom_of(headText, "head atom");
    r.nVars = sc.nextVar;
    return r;
}

Rule RuleParser::parse_json(const std::string& json) const {
    Scope sc;
    Rule r;
    auto term_of = [&](const std::string& tj) {
        std::string type = json_str(tj, "type");
        std::string value = json_str(tj, "value");
        if (value.empty()) throw RuleError("JSON term missing 'value': " + tj);
        if (type == "variable") return var_term(value, sc);
        std::string spelled;
        expand(value, spelled);
        return const_term(spelled, sc);
    };
    auto atom_of = [&](const std::string& aj) {
        size_t sp = aj.find("\"subject\"");
        std::string sj = json_object_at(aj, aj.find('{', sp));
        size_t op = aj.find("\"object\"");
        std::string oj = json_object_at(aj, aj.find('{', op));
        std::string ps = json_str(aj, "predicate");
        if (ps.empty()) throw RuleError("JSON atom missing 'predicate': " + aj);
        Atom a;
        a.s = term_of(sj);
        a.o = term_of(oj);
        a.pred = pred_id(ps);
        return a;
    };
    size_t bodyPos = json.find("\"body\"");
    size_t arrStart = json.find('[', bodyPos);
    if (bodyPos == std::string::npos || arrStart == std::string::npos) throw RuleError("JSON rule missing 'body' array");
    size_t arrEnd = json.find(']', arrStart);
    std::string arr = json.substr(arrStart + 1, arrEnd == std::string::npos ? std::string::npos : arrEnd - arrStart - 1);
    for (const auto& aj : json_objects(arr)) r.body.push_back(atom_of(aj));
    size_t headPos = json.find("\"head\"");
    if (headPos == std::string::npos) throw RuleError("JSON rule missing 'head'");
    r.head = atom_of(json_object_at(json, json.find('{', headPos)));
    r.nVars = sc.nextVar;
    return r;
}

}  // namespace gr
