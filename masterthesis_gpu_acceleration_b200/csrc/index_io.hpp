// index_io.hpp — a loaded graph (dictionaries, rule prefixes, host index)
// saved to and read back from one binary file, so that a graph is parsed
// and indexed once and later loads skip both.  The file holds exactly the
// arrays the index keeps, in this machine's byte order, after a header with
// a format version, and ends with a checksum of everything before it; a file
// of another version, with a wrong checksum or of inconsistent sizes is
// refused.
#pragma once
#include <string>
#include <unordered_map>

#include "index.hpp"
#include "turtle.hpp"

namespace gr {

using Prefixes = std::unordered_map<std::string, std::string>;

bool save_graph_file(const std::string& path, const TermDict& ents, const TermDict& preds,
                     const Prefixes& prefixes, const HostIndex& ix, std::string* err);

// Fills ents, preds, prefixes and ix (which should be empty) from a file
// written by save_graph_file.
bool load_graph_file(const std::string& path, TermDict& ents, TermDict& preds, Prefixes& prefixes,
                     HostIndex& ix, std::string* err);

}  // namespace gr
