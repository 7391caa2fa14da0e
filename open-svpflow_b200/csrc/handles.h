// handles.h -- read access to the public handles (defined in capi.cpp) for the other
// host translation units: the batch and serving runtimes and the allocation-free path.
#pragma once
#include <string>

#include "../../include/svpflow_b200.h"
#include "svpf_device.h"

namespace svpf {
const SuperOpts *super_opts_of(const svpf_super *s);
const SuperLayout *super_layout_of(const svpf_super *s);
const SuperDev *super_dev_of(const svpf_super *s);
const AnalyseOpts *analyser_opts(const svpf_analyser *a);
const AnalyseParams *analyser_params(const svpf_analyser *a);
const SuperLayout *analyser_layout(const svpf_analyser *a);
int32_t analyser_delta(const svpf_analyser *a);
void set_last_error(const std::string &msg);
void add_launches(int n);
// 0 when a CUDA device is usable, else SVPF_ECUDA with the message set
int require_device();
}  // namespace svpf
