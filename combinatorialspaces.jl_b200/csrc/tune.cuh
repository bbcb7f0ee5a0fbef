// The autotuner's table: the variant chosen per (kernel, dtype, shape, size bucket), shared by every
// handle in the process, consulted when a kernel is launched (or a graph captured) and saved to /
// loaded from a JSON file so a later process starts from the measured choices.
#pragma once
#include <string>

namespace decb {
// floor(log2(n)) for n >= 1 (0 for n < 1): the size bucket of a tuning key.
int size_bucket(long long n);
// The variant stored under key, or dflt if none was measured.
int tune_get(const std::string& key, int dflt);
void tune_set(const std::string& key, int value);
void tune_clear();
// Bumped by every change to the table, so launch sites can cache a lookup.
unsigned tune_version();
// JSON: {"format": "dec_b200 tuning table", "version": 1, "device": "...", "entries": {"key": value, ...}}
void tune_save(const std::string& path);
// Merges a saved table into the current one (entries in the file win); returns the entries read.
int tune_load(const std::string& path);
}  // namespace decb
