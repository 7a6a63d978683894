// rules.hpp — rule text / JSON front-end.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

#include "turtle.hpp"

namespace gr {

// A term is a variable (dense id, first-seen order) or a constant entity.
// Constants that name no entity of the graph get negative ids (unique per
// spelling within the rule); they match no triple.
struct Term {
    bool isVar = true;
    int32_t id = -1;
};

// pred < 0: the predicate names no predicate of the graph.
struct Atom {
    int32_t pred = -1;
    Term s, o;
};

struct Rule {
    Atom head;
    std::vector<Atom> body;
    int32_t nVars = 0;
};

struct RuleError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

class RuleParser {
public:
    RuleParser(const TermDict& ents, const TermDict& preds,
               std::unordered_map<std::string, std::string> prefixes)
        : ents_(ents), preds_(preds), prefixes_(std::move(prefixes)) {}

    // Text syntax of CPU_01_nonparallel/RuleParser.cpp:199-270:
    //   "(?a <p> ?b) ^ (?b pfx:q ?c) => (?a <r> ?c)"  — anything after '|' is ignored.
    Rule parse_text(const std::string& line) const;
    // RDFRules JSON export syntax of CPU_01_nonparallel/RuleParser.cpp:342-368.
    Rule parse_json(const std::string& json) const;

private:
    const TermDict& ents_;
    const TermDict& preds_;
    std::unordered_map<std::string, std::string> prefixes_;

    // The token's IRI as the dictionaries spell it ('<...>' stripped, a
    // known prefix expanded), written into `out`.
    void expand(std::string_view token, std::string& out) const;
    // Names seen in one rule: a handful, so searched linearly.
    struct Scope {
        std::vector<std::pair<std::string, int32_t>> vars;
        std::vector<std::pair<std::string, int32_t>> unknown;
        int32_t nextVar = 0;
    };
    Term var_term(std::string_view name, Scope& sc) const;
    Term const_term(const std::string& spelled, Scope& sc) const;
    Term text_term(std::string_view token, Scope& sc) const;
    int32_t pred_id(std::string_view token) const;
};

}  // namespace gr
