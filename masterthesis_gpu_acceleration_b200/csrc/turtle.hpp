// turtle.hpp — Turtle ingest and term dictionaries.
#pragma once
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

namespace gr {

// Dense ids for strings in first-seen order.
struct TermDict {
    std::unordered_map<std::string, int32_t> map;
    std::vector<std::string> names;
    int32_t intern(const std::string& s) {
        auto it = map.find(s);
        if (it != map.end()) return it->second;
        int32_t id = (int32_t)names.size();
        map.emplace(s, id);
        names.push_back(s);
        return id;
    }
    int32_t find(const std::string& s) const {
        auto it = map.find(s);
        return it == map.end() ? -1 : it->second;
    }
    size_t size() const { return names.size(); }
};

// Parses a Turtle file with the syntax subset the reference accepts
// (CPU_01_nonparallel/RdfIndexes.cpp:146-415): IRIs, prefixed names,
// @prefix / PREFIX, blank nodes, literals with language tags or datatypes,
// 'a', booleans, numbers, ';' and ',' lists.  Subjects and objects are
// interned in `ents`, predicates in `preds`; triples are appended to `spo`
// as (s, p, o) int32 triples (duplicates are kept; the index drops them).
bool parse_turtle_file(const std::string& path, TermDict& ents, TermDict& preds,
                       std::vector<int32_t>& spo, std::string* err);
bool parse_turtle_text(const std::string& text, TermDict& ents, TermDict& preds,
                       std::vector<int32_t>& spo);
// The same result (identical ids and triple order) read by several threads:
// the text is cut after statement ends into chunks of at least minChunk
// bytes, each read with the prefixes of the first chunk, and the chunks'
// dictionaries are merged in file order.  Texts with long literals ("""),
// anonymous nodes ([ ]) or prefix declarations after the first chunk are
// read by one reader.
bool parse_turtle_text_parallel(const std::string& text, TermDict& ents, TermDict& preds,
                                std::vector<int32_t>& spo, size_t minChunk = size_t(4) << 20);
bool read_file(const std::string& path, std::string& text, std::string* err);

// Prefix map the rule parser uses: a line-based scan for '@prefix' or
// 'prefix' lines with a non-empty name and IRI, as
// CPU_01_nonparallel/RuleParser.cpp:48-93 reads them.
std::unordered_map<std::string, std::string> scan_rule_prefixes(const std::string& path);
std::unordered_map<std::string, std::string> scan_rule_prefixes_text(const std::string& text);

}  // namespace gr
