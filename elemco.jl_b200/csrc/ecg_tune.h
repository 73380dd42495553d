// ecg_tune.h — the GEMM autotuner's table and its measurement helper.
//
// A launcher that has more than one valid configuration for a GEMM shape
// (tile shape, split-K count) looks the shape up in a process-wide table.  On
// a miss, with tuning enabled and the stream not capturing, it times every
// candidate on the call's own operands (each run twice, the second timed with
// CUDA events; the output is saved before and restored after each run, so the
// call's result is unaffected), records the fastest and runs it.  Without an
// entry and with tuning off the launcher's fixed rule applies.  The table can
// be saved to and loaded from a text file ("key value" lines).
#pragma once
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "ecg_dev.h"

namespace ecg {
namespace dev {

void set_tuning(bool on);
bool tuning();
bool tune_get(const std::string& key, int* value);
void tune_put(const std::string& key, int value);
size_t tune_size();
std::string tune_dump();                 // "key value\n" lines
int tune_parse(const std::string& text);  // returns entries read, -1 on a bad line
bool stream_capturing(stream_t s);

// The output region a candidate overwrites: ncols columns of rows_bytes bytes
// at C, ldc_bytes apart.
struct TuneOut {
  void* C;
  int64_t rows_bytes, ncols, ldc_bytes;
};
// Times each candidate (run(i) launches candidate i, returning 0 or a CUDA
// error) and returns the index of the fastest (-1 if none ran); the output
// region holds its original contents again afterwards.
int tune_pick(stream_t s, int ncand, const std::function<int(int)>& run, const TuneOut& out);

}  // namespace dev
}  // namespace ecg
