// nvrtc_module.cpp — compiles the per-driver kernel module (see header).
#include "nvrtc_module.hpp"

#include <nvrtc.h>

#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <dirent.h>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "../../include/mppi_b200/mppi_backend.h"

namespace mppi_b200 {

namespace {

struct EmbeddedFile {
  const char* name;
  const char* text;
};

#include "embedded_sources.inc"  // kEmbeddedFiles[] (generated by build.py)

uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ull) {
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

bool read_file(const std::string& path, std::string* out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::ostringstream ss;
  ss << f.rdbuf();
  *out = ss.str();
  return true;
}

std::string dir_of(const std::string& path) {
  const size_t p = path.find_last_of('/');
  return p == std::string::npos ? std::string(".") : path.substr(0, p);
}

// Contents of the headers next to the plugin (plugins include their own
// parameter-layout headers), so an edited header invalidates cached cubins.
std::string sibling_headers(const std::string& dir) {
  std::string acc;
  DIR* d = opendir(dir.c_str());
  if (!d) return acc;
  std::map<std::string, std::string> files;
  while (dirent* e = readdir(d)) {
    const std::string n = e->d_name;
    const auto ends = [&](const char* suf) {
      const size_t l = strlen(suf);
      return n.size() > l && n.compare(n.size() - l, l, suf) == 0;
    };
    if (ends(".h") || ends(".cuh") || ends(".hpp")) {
      std::string text;
      if (read_file(dir + "/" + n, &text)) files[n] = text;
    }
  }
  closedir(d);
  for (auto& kv : files) acc += kv.first + "\n" + kv.second;
  return acc;
}

std::string cache_dir() {
  if (const char* off = getenv("MPPI_B200_NO_DISK_CACHE"); off && *off && *off != '0') return "";
  if (const char* d = getenv("MPPI_B200_CACHE_DIR"); d && *d) return d;
  if (const char* x = getenv("XDG_CACHE_HOME"); x && *x) return std::string(x) + "/mppi_b200";
  if (const char* h = getenv("HOME"); h && *h) return std::string(h) + "/.cache/mppi_b200";
  return "";
}

void mkdirs(const std::string& path) {
  std::string cur;
  for (size_t i = 0; i < path.size(); ++i) {
    cur += path[i];
    if (path[i] == '/' && cur.size() > 1) mkdir(cur.c_str(), 0755);
  }
  mkdir(path.c_str(), 0755);
}

// Finds `identifier "<name>" is undefined` in an NVRTC log.
bool log_names_undefined(const std::string& log, const std::string& name) {
  if (name.empty()) return false;
  return log.find("identifier \"" + name + "\" is undefined") != std::string::npos;
}

std::mutex g_mutex;
std::map<uint64_t, std::shared_ptr<const KernelModule>> g_modules;

}  // namespace

bool valid_schema_hash(const std::string& s) {
  if (s.size() > 256) return false;
  for (char c : s)
    if (c < 0x20 || c > 0x7e || c == '"' || c == '\\') return false;
  return true;
}

const char* embedded_source(const char* name) {
  for (const auto& f : kEmbeddedFiles)
    if (strcmp(f.name, name) == 0) return f.text;
  return nullptr;
}

namespace {

struct CompileResult {
  uint64_t key = 0;
  std::string cubin;
  std::string log;
};

// Builds the NVRTC program for `spec` and compiles it to an sm_100a cubin
// (or fetches it from the on-disk cache).  Needs no GPU.
int compile_module(const ModuleSpec& spec, bool use_cache, bool ptxas_verbose,
                   CompileResult* res, std::string* error) {
  // ---- plugin source (metal_backend.mm:278-293: load the user library) ----
  if (spec.plugin_path.empty()) {
    *error = "user_metallib_path is empty.";
    return MPPI_ERR_PLUGIN;
  }
  std::string plugin_text;
  if (!read_file(spec.plugin_path, &plugin_text)) {
    *error = "Failed to load user plugin source '" + spec.plugin_path +
             "': file not found or unreadable.";
    return MPPI_ERR_PLUGIN;
  }

  const std::string stage = spec.stage_cost.empty() ? "mppi_default_stage_cost" : spec.stage_cost;
  const std::string term =
      spec.terminal_cost.empty() ? "mppi_default_terminal_cost" : spec.terminal_cost;
  std::vector<std::string> opts = {
      "--gpu-architecture=sm_100a",
      "-std=c++17",
      "-lineinfo",
      "--include-path=" + dir_of(spec.plugin_path),
      "-DMPPI_STATE_DIM=" + std::to_string(spec.state_dim),
      // the state buffer: the reference's 128 bytes, or the state's size
      "-DMPPI_MAX_STATE_BYTES=" +
          std::to_string(std::max<uint64_t>(128, ((uint64_t)spec.state_dim * 4 + 15) / 16 * 16)),
      "-DMPPI_CONTROL_DIM=" + std::to_string(spec.control_dim),
      "-DMPPI_COV_FULL=" + std::to_string(spec.cov_full ? 1 : 0),
      "-DMPPI_CONTROL_COST=" + std::to_string(spec.control_cost ? 1 : 0),
      "-DMPPI_NOISE_HALF=" + std::to_string(spec.noise_half ? 1 : 0),
      "-DMPPI_MP_BYTES=" + std::to_string(spec.model_params_bytes),
      "-DMPPI_CP_BYTES=" + std::to_string(spec.cost_params_bytes),
      "-DMPPI_DYNAMICS_FN=" + spec.dynamics,
      "-DMPPI_STAGE_COST_FN=" + stage,
      "-DMPPI_TERMINAL_COST_FN=" + term,
      "-DMPPI_PROPOSAL=" + std::to_string(spec.proposal ? 1 : 0),
      "-DMPPI_MP_ALIGN=" + std::to_string(spec.model_params_alignment ? spec.model_params_alignment : 1),
      "-DMPPI_CP_ALIGN=" + std::to_string(spec.cost_params_alignment ? spec.cost_params_alignment : 1),
      "-DMPPI_SCHEMA_HASH=\"" + spec.schema_hash + "\"",
  };
  if (!valid_schema_hash(spec.schema_hash)) {
    *error = "ParamLayout::schema_hash must be printable ASCII without quotes or backslashes "
             "(at most 256 characters).";
    return MPPI_ERR_INVALID;
  }
  if (!spec.features.empty()) opts.push_back("-DMPPI_FEATURES_FN=" + spec.features);
  if (ptxas_verbose) opts.push_back("--ptxas-options=-v");

  const std::string main_src = "#include \"mppi_prelude.cuh\"\n#line 1 \"" + spec.plugin_path +
                               "\"\n" + plugin_text +
                               "\n#line 1 \"mppi_kernels.cuh\"\n#include \"mppi_kernels.cuh\"\n";
  static const char* kShim = "#pragma once\n#include \"mppi_prelude.cuh\"\n";
  std::vector<const char*> hdr_text, hdr_name;
  for (const auto& f : kEmbeddedFiles) {
    hdr_name.push_back(f.name);
    hdr_text.push_back(f.text);
  }
  // The reference's plugin headers, so MSL-style includes resolve.
  hdr_name.push_back("mppi_core.h");
  hdr_text.push_back(kShim);
  hdr_name.push_back("philox.h");
  hdr_text.push_back(kShim);

  int nv_major = 0, nv_minor = 0;
  nvrtcVersion(&nv_major, &nv_minor);
  std::string key_material = main_src + sibling_headers(dir_of(spec.plugin_path));
  for (size_t i = 0; i < hdr_name.size(); ++i) key_material += hdr_name[i] + std::string(hdr_text[i]);
  for (const auto& o : opts) key_material += "\n" + o;
  key_material += "\nnvrtc " + std::to_string(nv_major) + "." + std::to_string(nv_minor);
  res->key = fnv1a(key_material);

  const std::string cdir = use_cache ? cache_dir() : "";
  char hexkey[32];
  snprintf(hexkey, sizeof(hexkey), "%016llx", (unsigned long long)res->key);
  const std::string cpath = cdir.empty() ? "" : cdir + "/" + hexkey + ".cubin";
  if (!cpath.empty() && read_file(cpath, &res->cubin) && !res->cubin.empty()) return MPPI_OK;
  res->cubin.clear();

  nvrtcProgram prog;
  nvrtcResult r = nvrtcCreateProgram(&prog, main_src.c_str(), "mppi_module.cu",
                                     (int)hdr_name.size(), hdr_text.data(), hdr_name.data());
  if (r != NVRTC_SUCCESS) {
    *error = std::string("nvrtcCreateProgram failed: ") + nvrtcGetErrorString(r);
    return MPPI_ERR_PLUGIN;
  }
  std::vector<const char*> copts;
  for (const auto& o : opts) copts.push_back(o.c_str());
  r = nvrtcCompileProgram(prog, (int)copts.size(), copts.data());
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  std::string log(log_size, '\0');
  if (log_size > 1) nvrtcGetProgramLog(prog, &log[0]);
  res->log = log;
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    // metal_backend.mm:295-334: a missing callable is named in the error.
    if (log_names_undefined(log, spec.dynamics)) {
      *error = "Required callable '" + spec.dynamics + "' not found in user plugin source '" +
               spec.plugin_path + "'.";
      return MPPI_ERR_CALLABLE;
    }
    for (const std::string* nm : {&spec.stage_cost, &spec.terminal_cost, &spec.features}) {
      if (log_names_undefined(log, *nm)) {
        *error = "Callable '" + *nm + "' not found in user plugin source '" + spec.plugin_path +
                 "'.";
        return MPPI_ERR_CALLABLE;
      }
    }
    // ParamLayout against the plugin's MPPI_PARAM_LAYOUT: name the field
    const std::string marker = "MPPI_PARAM_LAYOUT_MISMATCH: ";
    const size_t at = log.find(marker);
    if (at != std::string::npos) {
      const size_t from = at + marker.size();
      const size_t to = log.find('"', from);
      *error = "Declared parameter layout does not match the plugin '" + spec.plugin_path +
               "': " + log.substr(from, to == std::string::npos ? std::string::npos : to - from) +
               " (MPPI_PARAM_LAYOUT).";
      return MPPI_ERR_INVALID;
    }
    *error = "Failed to compile user plugin '" + spec.plugin_path + "' with the MPPI kernels:\n" +
             log;
    return MPPI_ERR_PLUGIN;
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  res->cubin.resize(n);
  nvrtcGetCUBIN(prog, &res->cubin[0]);
  nvrtcDestroyProgram(&prog);
  if (!cpath.empty()) {
    mkdirs(cdir);
    const std::string tmp = cpath + ".tmp." + std::to_string(getpid());
    std::ofstream f(tmp, std::ios::binary);
    if (f) {
      f.write(res->cubin.data(), (std::streamsize)res->cubin.size());
      f.close();
      rename(tmp.c_str(), cpath.c_str());
    }
  }
  return MPPI_OK;
}

}  // namespace

int compile_check(const ModuleSpec& spec, std::string* log, std::string* error) {
  CompileResult res;
  const int rc = compile_module(spec, false, true, &res, error);
  *log = res.log;
  return rc;
}

int load_module(const ModuleSpec& spec, std::shared_ptr<const KernelModule>* out,
                std::string* error) {
  std::lock_guard<std::mutex> lock(g_mutex);
  CompileResult res;
  const bool verbose = getenv("MPPI_B200_PTXAS_VERBOSE") && *getenv("MPPI_B200_PTXAS_VERBOSE") == '1';
  if (int rc = compile_module(spec, true, verbose, &res, error)) return rc;
  if (auto it = g_modules.find(res.key); it != g_modules.end()) {
    *out = it->second;
    return MPPI_OK;
  }
  auto mod = std::make_shared<KernelModule>();
  mod->build_log = res.log;
  cudaError_t ce = cudaLibraryLoadData(&mod->library, res.cubin.data(), nullptr, nullptr, 0,
                                       nullptr, nullptr, 0);
  if (ce != cudaSuccess) {
    *error = std::string("cudaLibraryLoadData failed: ") + cudaGetErrorString(ce);
    cudaGetLastError();
    return ce == cudaErrorNoDevice || ce == cudaErrorInsufficientDriver ? MPPI_ERR_NO_DEVICE
                                                                         : MPPI_ERR_CUDA;
  }
  const char* names[3] = {"mppi_rollout_b64", "mppi_rollout_b128", "mppi_rollout_b256"};
  const char* fused_names[3] = {"mppi_rollout_fused_b64", "mppi_rollout_fused_b128",
                                "mppi_rollout_fused_b256"};
  for (int i = 0; i < 3; ++i) {
    ce = cudaLibraryGetKernel(&mod->rollout[i], mod->library, names[i]);
    if (ce == cudaSuccess) ce = cudaLibraryGetKernel(&mod->rollout_fused[i], mod->library,
                                                     fused_names[i]);
    if (ce != cudaSuccess) break;
  }
  if (ce == cudaSuccess)
    ce = cudaLibraryGetKernel(&mod->rollout_work, mod->library, "mppi_rollout_work_b128");
  if (ce == cudaSuccess)
    ce = cudaLibraryGetKernel(&mod->rollout_work_fused, mod->library,
                              "mppi_rollout_work_fused_b128");
  if (ce == cudaSuccess)
    ce = cudaLibraryGetKernel(&mod->rollout_early, mod->library, "mppi_rollout_early_b128");
  if (ce == cudaSuccess)
    ce = cudaLibraryGetKernel(&mod->rollout_early_fused, mod->library,
                              "mppi_rollout_early_fused_b128");
  if (ce == cudaSuccess) ce = cudaLibraryGetKernel(&mod->rollout_ws, mod->library, "mppi_rollout_ws_b128");
  if (ce == cudaSuccess)
    ce = cudaLibraryGetKernel(&mod->rollout_ws_fused, mod->library, "mppi_rollout_ws_fused_b128");
  if (ce == cudaSuccess)
    ce = cudaLibraryGetKernel(&mod->rollout_coop[0], mod->library, "mppi_rollout_coop32");
  if (ce == cudaSuccess)
    ce = cudaLibraryGetKernel(&mod->rollout_coop_fused[0], mod->library,
                              "mppi_rollout_coop32_fused");
  if (ce == cudaSuccess)
    ce = cudaLibraryGetKernel(&mod->rollout_coop[1], mod->library, "mppi_rollout_coop");
  if (ce == cudaSuccess)
    ce = cudaLibraryGetKernel(&mod->rollout_coop_fused[1], mod->library, "mppi_rollout_coop_fused");
  if (ce == cudaSuccess) {
    // lanes per sample of the cooperative form (0: the plugin declares no split)
    void* g = nullptr;
    size_t gs = 0;
    ce = cudaLibraryGetGlobal(&g, &gs, mod->library, "mppi_coop_lanes");
    if (ce == cudaSuccess && gs == sizeof(uint32_t))
      ce = cudaMemcpy(&mod->coop_lanes, g, sizeof(uint32_t), cudaMemcpyDeviceToHost);
  }
  if (ce == cudaSuccess) ce = cudaLibraryGetKernel(&mod->combine, mod->library, "mppi_combine");
  if (ce == cudaSuccess) ce = cudaLibraryGetKernel(&mod->weights, mod->library, "mppi_weights");
  if (ce == cudaSuccess) ce = cudaLibraryGetKernel(&mod->noise, mod->library, "mppi_noise");
  if (ce == cudaSuccess && !spec.features.empty())
    ce = cudaLibraryGetKernel(&mod->features, mod->library, "mppi_features");
  if (ce == cudaSuccess && !spec.features.empty())
    ce = cudaLibraryGetKernel(&mod->proposal_rows, mod->library, "mppi_proposal_rows");
  for (int i = 0; i < 3 && ce == cudaSuccess; ++i) {
    cudaFuncAttributes fa{}, ff{};
    ce = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(mod->rollout[i]));
    if (ce == cudaSuccess)
      ce = cudaFuncGetAttributes(&ff, reinterpret_cast<const void*>(mod->rollout_fused[i]));
    mod->rollout_static_smem[i] = std::max(fa.sharedSizeBytes, ff.sharedSizeBytes);
  }
  if (ce == cudaSuccess) {
    // the early-noise 128-sample forms share the 128-sample geometry
    cudaFuncAttributes fa{}, ff{};
    ce = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(mod->rollout_early));
    if (ce == cudaSuccess)
      ce = cudaFuncGetAttributes(&ff, reinterpret_cast<const void*>(mod->rollout_early_fused));
    mod->rollout_static_smem[1] =
        std::max(mod->rollout_static_smem[1], std::max(fa.sharedSizeBytes, ff.sharedSizeBytes));
  }
  if (ce == cudaSuccess) {
    cudaFuncAttributes fa{}, ff{};
    ce = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(mod->rollout_ws));
    if (ce == cudaSuccess)
      ce = cudaFuncGetAttributes(&ff, reinterpret_cast<const void*>(mod->rollout_ws_fused));
    mod->ws_static_smem = std::max(fa.sharedSizeBytes, ff.sharedSizeBytes);
  }
  for (int v = 0; v < 2 && ce == cudaSuccess; ++v) {
    cudaFuncAttributes fa{}, ff{};
    ce = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(mod->rollout_coop[v]));
    if (ce == cudaSuccess)
      ce = cudaFuncGetAttributes(&ff, reinterpret_cast<const void*>(mod->rollout_coop_fused[v]));
    mod->coop_static_smem[v] = std::max(fa.sharedSizeBytes, ff.sharedSizeBytes);
  }
  if (ce == cudaSuccess) {
    cudaFuncAttributes fa{}, ff{};
    ce = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(mod->rollout_work));
    if (ce == cudaSuccess)
      ce = cudaFuncGetAttributes(&ff, reinterpret_cast<const void*>(mod->rollout_work_fused));
    mod->work_static_smem = std::max(fa.sharedSizeBytes, ff.sharedSizeBytes);
  }
  if (ce != cudaSuccess) {
    *error = std::string("Required library kernel missing from the module: ") +
             cudaGetErrorString(ce);
    cudaGetLastError();
    return MPPI_ERR_CUDA;
  }
  g_modules[res.key] = mod;
  *out = mod;
  return MPPI_OK;
}

}  // namespace mppi_b200
