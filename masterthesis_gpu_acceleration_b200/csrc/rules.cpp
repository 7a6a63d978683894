// rules.cpp — rule text / JSON front-end with the reference's accepted syntax.
#include "rules.hpp"

#include <cctype>

namespace gr {
namespace {

std::string trim(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
}

// The first three whitespace-separated tokens of s, as
// `istringstream(s) >> a >> b >> c` reads them (RuleParser.cpp reads an atom
// that way): leading whitespace skipped, missing tokens left empty, anything
// after the third ignored.
void three_tokens(const std::string& s, std::string& a, std::string& b, std::string& c) {
    std::string* out[3] = {&a, &b, &c};
    size_t i = 0;
    const size_t n = s.size();
    for (std::string* t : out) {
        while (i < n && std::isspace((unsigned char)s[i])) ++i;
        size_t j = i;
        while (j < n && !std::isspace((unsigned char)s[j])) ++j;
        t->assign(s, i, j - i);
        i = j;
    }
}

// Splits the body on '^' outside parentheses (RuleParser.cpp:155-184).
std::vector<std::string> split_atoms(const std::string& body) {
    std::vector<std::string> out;
    std::string cur;
    int depth = 0;
    for (char ch : body) {
        if (ch == '(') { ++depth; cur.push_back(ch); }
        else if (ch == ')') { --depth; cur.push_back(ch); }
        else if (ch == '^' && depth == 0) {
            std::string t = trim(cur);
            if (!t.empty()) out.push_back(t);
            cur.clear();
        } else cur.push_back(ch);
    }
    std::string t = trim(cur);
    if (!t.empty()) out.push_back(t);
    return out;
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

std::string RuleParser::expand(const std::string& token) const {
    if (token.empty()) return token;
    if (token.front() == '<' && token.back() == '>') return token.substr(1, token.size() - 2);
    if (token.front() == '?' || token.front() == '"') return token;
    size_t c = token.find(':');
    if (c == std::string::npos) return token;
    auto it = prefixes_.find(token.substr(0, c));
    if (it != prefixes_.end()) return it->second + token.substr(c + 1);
    return token;
}

Term RuleParser::var_term(const std::string& name, Scope& sc) const {
    Term t;
    t.isVar = true;
    for (const auto& v : sc.vars)
        if (v.first == name) { t.id = v.second; return t; }
    t.id = sc.nextVar++;
    sc.vars.emplace_back(name, t.id);
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

Term RuleParser::text_term(const std::string& token, Scope& sc) const {
    std::string c = trim(token);
    if (c.empty()) throw RuleError("Empty term token");
    if (c.front() == '?') return var_term(c, sc);
    return const_term(expand(c), sc);
}

int32_t RuleParser::pred_id(const std::string& token) const {
    return preds_.find(expand(token));
}

Rule RuleParser::parse_text(const std::string& line) const {
    std::string clean = trim(line);
    if (clean.empty()) throw RuleError("Empty rule line");
    size_t bar = clean.find('|');
    if (bar != std::string::npos) clean = trim(clean.substr(0, bar));
    size_t arrow = clean.find("=>");
    if (arrow == std::string::npos) throw RuleError("Rule line missing => : " + line);
    std::string bodyText = trim(clean.substr(0, arrow));
    std::string headText = trim(clean.substr(arrow + 2));
    Scope sc;
    Rule r;
    auto atom_of = [&](const std::string& raw, const char* what) {
        std::string s = trim(raw);
        if (s.empty() || s.front() != '(' || s.back() != ')') throw RuleError(std::string("Invalid ") + what + ": " + raw);
        std::string st, pt, ot;
        three_tokens(s.substr(1, s.size() - 2), st, pt, ot);
        if (st.empty() || pt.empty() || ot.empty()) throw RuleError(std::string("Invalid ") + what + ": " + raw);
        Atom a;
        a.s = text_term(st, sc);
        a.o = text_term(ot, sc);
        a.pred = pred_id(pt);
        return a;
    };
    for (const auto& a : split_atoms(bodyText)) r.body.push_back(atom_of(a, "body atom"));
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
        return const_term(expand(value), sc);
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
