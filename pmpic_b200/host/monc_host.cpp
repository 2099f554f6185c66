// monc_host.cpp -- a C++ host for the B200 hot path that mirrors the
// reference's MONC component framework (pmpic_monc executable).
//
// Reference interfaces mirrored:
//   component descriptor  model_core/src/components/monc_component.F90:51-107
//                         (name, version, initialisation / timestep /
//                          finalisation callbacks taking the model state)
//   registry              model_core/src/components/registry.F90:101-131
//                         (<name>_enabled options), :285-292 (timestep
//                         callbacks of a group), :307-332 (group ordering)
//   timestepper           model_core/src/components/timestepper.F90:29-106
//                         (groups of type entire / rk_integrated; an RK group
//                          runs rksteps times per step)
//   options database      model_core/src/configuration/configurationfileparser.F90:26-329
//                         (key=value, # comments, global_configuration=
//                          include, += list append, --key=value overrides
//                          applied after the file), optionsdatabase.F90
//   model loop            model_core/src/monc.F90:200-235 (perform_model_steps;
//                         termination on nn_timesteps / termination_time,
//                         components/terminationcheck/src/terminationcheck.F90:91-147)
// The five hot-path components call the C ABI of include/pmpic_gpu.h; errors
// end the run like the reference's `error stop` (non-zero exit).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/pmpic_gpu.h"

namespace monc {

// ---- options database ----------------------------------------------------------
class Options {
 public:
  std::map<std::string, std::string> kv;

  static std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? "" : s.substr(a, b - a + 1);
  }
  static std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
  }
  // one key=value or key+=value line (comments after '#')
  bool apply_line(const std::string& raw, const std::string& dir, int depth, std::string* err) {
    std::string line = raw.substr(0, raw.find('#'));
    line = trim(line);
    if (line.empty()) return true;
    bool append = false;
    size_t eq = line.find("+=");
    if (eq != std::string::npos) {
      append = true;
    } else {
      eq = line.find('=');
      if (eq == std::string::npos) return true;
    }
    std::string key = lower(trim(line.substr(0, eq)));
    std::string val = trim(line.substr(eq + (append ? 2 : 1)));
    if (val.size() >= 2 && val.front() == '"' && val.back() == '"') val = val.substr(1, val.size() - 2);
    if (key == "global_configuration")
      return load(dir.empty() || (!val.empty() && val[0] == '/') ? val : dir + "/" + val, depth + 1, err);
    if (append && kv.count(key) && !kv[key].empty())
      kv[key] += "," + val;
    else
      kv[key] = val;
    return true;
  }
  bool load(const std::string& path, int depth, std::string* err) {
    if (depth > 8) {
      *err = "global_configuration nesting too deep";
      return false;
    }
    std::ifstream f(path);
    if (!f) {
      *err = "cannot read configuration file " + path;
      return false;
    }
    std::string dir = path.find('/') == std::string::npos ? "" : path.substr(0, path.rfind('/'));
    std::string line;
    while (std::getline(f, line))
      if (!apply_line(line, dir, depth, err)) return false;
    return true;
  }
  bool has(const std::string& k) const { return kv.count(lower(k)) > 0; }
  std::string str(const std::string& k, const std::string& d = "") const {
    auto it = kv.find(lower(k));
    return it == kv.end() ? d : it->second;
  }
  double real(const std::string& k, double d = 0.0) const {
    std::string s = str(k);
    if (s.empty()) return d;
    for (char& c : s)
      if (c == 'd' || c == 'D') c = 'e';  // Fortran exponent
    return std::atof(s.c_str());
  }
  long long integer(const std::string& k, long long d = 0) const {
    std::string s = str(k);
    return s.empty() ? d : std::atoll(s.c_str());
  }
  bool logical(const std::string& k, bool d = false) const {
    std::string s = lower(str(k));
    if (s.empty()) return d;
    return s == ".true." || s == "true" || s == "t" || s == "1";
  }
  std::vector<std::string> list(const std::string& k) const {
    std::vector<std::string> out;
    std::stringstream ss(str(k));
    std::string item;
    while (std::getline(ss, item, ',')) {
      item = lower(trim(item));
      if (!item.empty()) out.push_back(item);
    }
    return out;
  }
};

// ---- model state (the parts this host needs) -----------------------------------
struct State {
  Options options;
  pmpic_ctx* gpu = nullptr;
  int rksteps = 0;
  long long timestep = 0;
  long long iterations = 0;  // steps completed (state.F90:53)
  double time = 0.0;
  double dtm = 0.0;
  bool continue_timestep = true;
  pmpic_step_info info{};
  bool dry_run = false;
  std::vector<std::string> trace;  // callback order (dry runs)
};

using Callback = std::function<int(State&)>;

struct ComponentDescriptor {
  std::string name;
  float version = 0.1f;
  Callback initialisation, timestep, finalisation;
};

static int check(State& s, int rc, const char* what) {
  if (rc != 0) {
    std::fprintf(stderr, "error in %s: %d (%s)\n", what, rc, s.gpu ? pmpic_last_error(s.gpu) : "");
  }
  return rc;
}

// ---- the five hot-path components + set-up and control --------------------------
static ComponentDescriptor gpu_component(const char* name, int (*fn)(pmpic_ctx*)) {
  ComponentDescriptor d;
  d.name = name;
  d.timestep = [fn, name](State& s) {
    if (s.dry_run) {
      s.trace.push_back(name);
      return 0;
    }
    int rc = check(s, fn(s.gpu), name);
    if (rc) return rc;
    rc = check(s, pmpic_get_step_info(s.gpu, &s.info), "pmpic_get_step_info");
    s.dtm = s.info.dtm;
    return rc;
  };
  return d;
}

// The device context: the grid (setup_grid.F90:45-104) and the parcel store of
// max_parcels (parcelsetup_base.F90:49-81), created by the first component
// that needs it (parcelsetup_base, a set-up component or an integrator).
static int ensure_context(State& s) {
  if (s.gpu || s.dry_run) return 0;
  const Options& o = s.options;
  pmpic_config cfg{};
  cfg.nx = (int32_t)o.integer("nx");
  cfg.ny = (int32_t)o.integer("ny");
  cfg.nz = (int32_t)o.integer("nz");
  cfg.xmin = o.real("xmin");
  cfg.xmax = o.real("xmax");
  cfg.ymin = o.real("ymin");
  cfg.ymax = o.real("ymax");
  cfg.zmin = o.real("zmin");
  cfg.zmax = o.real("zmax");
  cfg.dtm = o.real("dtm");
  cfg.dtmax = o.real("dtmax", cfg.dtm);
  cfg.timestep_prefactor = o.real("timestep_prefactor", 0.5);
  cfg.max_parcels = o.integer("max_parcels");
  cfg.precision = PMPIC_FP64;
  cfg.device = (int32_t)o.integer("device", 0);
  int rc = pmpic_create(&cfg, &s.gpu);
  if (rc) {
    std::fprintf(stderr, "pmpic_create failed: %d\n", rc);
    return rc;
  }
  s.dtm = cfg.dtm;
  // timer_mod (timer.F90:110-245): per-routine device times when timing_enabled
  if (o.logical("timing_enabled", false)) return check(s, pmpic_timing(s.gpu, 1), "pmpic_timing");
  return 0;
}
static int release_context(State& s) {
  if (s.gpu && s.options.logical("timing_enabled", false)) {
    std::printf("%-20s %12s %10s\n", "routine", "total ms", "calls");
    for (int id = 0; id < pmpic_timer_count(); ++id) {
      double ms = 0.0;
      int64_t calls = 0;
      if (pmpic_timer_read(s.gpu, id, &ms, &calls) == 0 && calls > 0)
        std::printf("%-20s %12.3f %10lld\n", pmpic_timer_name(id), ms, (long long)calls);
    }
  }
  if (s.gpu) pmpic_destroy(s.gpu);
  s.gpu = nullptr;
  return 0;
}

// an integrator's initialisation: one integrator only (rk4_integrator.F90:47-51,
// euler_integrator.F90:44-50), then the device context
static int integrator_init(State& s, int rksteps, const char* name) {
  if (s.rksteps != 0) {
    std::fprintf(stderr, "Error - another integrator component is present (%s). ABORTING\n", name);
    return (int)PMPIC_ERR_CONFIG;
  }
  s.rksteps = rksteps;
  return ensure_context(s);
}

// writebinary (writebinary.F90:31-134) and writenetcdf (writenetcdf.F90:84-180):
// <name>_mode none | step | time; files every <what>_step_write<sfx>_frequency
// steps (by the iteration count) or every <what>_time_write<sfx>_frequency of
// model time
static ComponentDescriptor writer(const char* name, bool netcdf) {
  struct Cfg {
    std::string mode;
    long long psteps = 0, gsteps = 0;
    double dtp = 0, dtg = 0, tnextp = 0, tnextg = 0;
  };
  auto c = std::make_shared<Cfg>();
  ComponentDescriptor d;
  d.name = name;
  const std::string sfx = netcdf ? "_netcdf" : "";
  d.initialisation = [c, sfx, name](State& s) {
    const Options& o = s.options;
    c->mode = Options::lower(o.str(std::string(name) + "_mode", "none"));
    if (c->mode == "time") {
      c->dtp = o.real("parcel_time_write" + sfx + "_frequency");
      c->dtg = o.real("grid_time_write" + sfx + "_frequency");
    } else if (c->mode == "step") {
      c->psteps = o.integer("parcel_step_write" + sfx + "_frequency");
      c->gsteps = o.integer("grid_step_write" + sfx + "_frequency");
    } else if (c->mode != "none") {
      std::fprintf(stderr, "Error: mode '%s' not recognised. The valid options are 'none', 'time' or 'step'\n",
                   c->mode.c_str());
      return (int)PMPIC_ERR_CONFIG;
    }
    return 0;
  };
  d.timestep = [c, netcdf, name](State& s) {
    if (s.dry_run) {
      s.trace.push_back(name);
      return 0;
    }
    const long long num = s.iterations;
    bool parcels = false, grids = false;
    if (c->mode == "step") {
      parcels = c->psteps != 0 && num % c->psteps == 0;
      grids = c->gsteps != 0 && num % c->gsteps == 0;
    } else if (c->mode == "time") {
      if (c->dtg != 0. && s.time >= c->tnextg) {
        grids = true;
        c->tnextg += c->dtg;
      }
      if (c->dtp != 0. && s.time >= c->tnextp) {
        parcels = true;
        c->tnextp += c->dtp;
      }
    }
    char path[64];
    int rc = 0;
    if (grids) {  // writebinary.F90:259, writenetcdf.F90:206
      if (netcdf) {
        std::snprintf(path, sizeof path, "grids_%04lld.nc", num);
        rc = check(s, pmpic_write_grids_netcdf(s.gpu, path, s.time + s.dtm, (int32_t)s.timestep), path);
      } else {
        std::snprintf(path, sizeof path, "grids_%05d_%05lld.dat", 0, num);
        rc = check(s, pmpic_write_grids(s.gpu, path, s.time), path);
      }
    }
    if (!rc && parcels) {  // writebinary.F90:160, writenetcdf.F90:333
      std::snprintf(path, sizeof path, netcdf ? "parcels_%05d_%05lld.nc" : "parcels_%05d_%05lld.dat", 0, num);
      rc = netcdf ? check(s, pmpic_write_parcels_netcdf(s.gpu, path, s.time + s.dtm, (int32_t)s.timestep), path)
                  : check(s, pmpic_write_parcels(s.gpu, path, s.time), path);
    }
    return rc;
  };
  return d;
}

static std::vector<ComponentDescriptor> all_components() {
  std::vector<ComponentDescriptor> v;
  ComponentDescriptor base;
  base.name = "parcelsetup_base";
  base.initialisation = ensure_context;
  base.finalisation = release_context;
  v.push_back(base);
  ComponentDescriptor rk4 = gpu_component("rk4_integrator", pmpic_rk4_integrator);
  rk4.initialisation = [](State& s) { return integrator_init(s, 4, "rk4_integrator"); };  // rk4_integrator.F90:51
  rk4.finalisation = release_context;
  ComponentDescriptor euler = gpu_component("euler_integrator", pmpic_euler_integrator);
  euler.initialisation = [](State& s) { return integrator_init(s, 1, "euler_integrator"); };  // :49
  v.push_back(euler);
  // prescribed_parcel_velocity (velocity.F90:58-262): quadrant tags at the
  // start of a run, then the analytic tendencies of velocity_profile each call
  ComponentDescriptor pv;
  pv.name = "prescribed_parcel_velocity";
  pv.initialisation = [](State& s) {
    const long long profile = s.options.integer("velocity_profile", -1);
    if (profile < PMPIC_VELOCITY_SHEAR || profile > PMPIC_VELOCITY_EVACUATE) {
      std::fprintf(stderr, "prescribed_parcel_velocity: velocity_profile %lld is not one of 0..10\n", profile);
      return (int)PMPIC_ERR_CONFIG;
    }
    if (s.dry_run) return 0;
    int rc = ensure_context(s);
    if (!rc && s.iterations == 0) rc = check(s, pmpic_prescribed_velocity_tag(s.gpu), "prescribed_velocity_tag");
    return rc;
  };
  pv.timestep = [](State& s) {
    if (s.dry_run) {
      s.trace.push_back("prescribed_parcel_velocity");
      return 0;
    }
    return check(s, pmpic_prescribed_velocity(s.gpu, (int)s.options.integer("velocity_profile")),
                 "prescribed_velocity");
  };
  v.push_back(pv);
  // basic_parcelsetup (basic_parcelsetup.F90:22-134), written on the device
  ComponentDescriptor basic;
  basic.name = "basic_parcelsetup";
  basic.initialisation = [](State& s) {
    if (s.dry_run) return 0;
    int rc = ensure_context(s);
    if (rc) return rc;
    return check(s, pmpic_setup_basic(s.gpu, (int32_t)s.options.integer("parcels_per_cell_dir")), "basic_parcelsetup");
  };
  v.push_back(basic);
  // plume_parcelsetup (plume_parcelsetup.F90:58-334), written on the device
  ComponentDescriptor plume;
  plume.name = "plume_parcelsetup";
  plume.initialisation = [](State& s) {
    const Options& o = s.options;
    pmpic_plume_params p{};
    p.lambda = o.real("lambda");
    p.H = o.real("h");
    p.z_c = o.real("z_c");
    p.mu = o.real("mu");
    p.z_d = o.real("z_d");
    p.z_m = o.real("z_m");
    p.r_plume = o.real("r_plume");
    const std::vector<std::string> e = o.list("e_values");
    if (e.size() != 3) {
      std::fprintf(stderr, "plume_parcelsetup: e_values needs 3 values\n");
      return (int)PMPIC_ERR_CONFIG;
    }
    for (int i = 0; i < 3; ++i) p.e_values[i] = std::atof(e[i].c_str());
    if (s.dry_run) return 0;
    int rc = ensure_context(s);
    if (rc) return rc;
    int64_t n_plume = 0;
    rc = check(s, pmpic_setup_plume(s.gpu, &p, &n_plume), "plume_parcelsetup");
    if (!rc) {
      int64_t n = 0;
      pmpic_get_count(s.gpu, &n);
      std::printf("Total number of parcels= %lld background= %lld plume= %lld\n", (long long)n,
                  (long long)(n - n_plume), (long long)n_plume);
    }
    return rc;
  };
  v.push_back(plume);
  // readfromfile_parcelsetup (readfromfile_parcelsetup.F90:26-130): restart
  // from the parcel dumps of step restart_num, every rank's file appended in
  // rank order; the dump's time becomes the model time
  ComponentDescriptor restart;
  restart.name = "readfromfile_parcelsetup";
  restart.initialisation = [](State& s) {
    const long long num = s.options.integer("restart_num");
    s.iterations = num;  // :43
    std::vector<std::string> files;
    for (int rank = 0;; ++rank) {  // :50-68
      char path[64];
      std::snprintf(path, sizeof path, "parcels_%05d_%05lld.dat", rank, num);
      std::ifstream f(path);
      if (!f) break;
      files.push_back(path);
    }
    if (files.empty()) {
      std::fprintf(stderr, "there is no file to restart from (parcels_00000_%05lld.dat)\n", num);
      return (int)PMPIC_ERR_CONFIG;
    }
    std::printf("Found %zu files\n", files.size());
    if (s.dry_run) return 0;
    int rc = ensure_context(s);
    for (size_t r = 0; r < files.size() && !rc; ++r) {  // :111-117
      double t = 0.0;
      rc = check(s, pmpic_read_parcels(s.gpu, files[r].c_str(), r > 0 ? 1 : 0, &t), files[r].c_str());
      if (!rc) s.time = t;  // read_file :220
    }
    return rc;
  };
  v.push_back(restart);
  v.push_back(writer("writebinary", false));
  v.push_back(writer("writenetcdf", true));
  v.push_back(gpu_component("vort2vel", pmpic_vort2vel));
  v.push_back(gpu_component("vorticity_tendency", pmpic_vorticity_tendency));
  v.push_back(rk4);
  v.push_back(gpu_component("parcel_splitting", pmpic_parcel_splitting));
  v.push_back(gpu_component("parcel_mixing", pmpic_parcel_mixing));
  // thermal_parcelsetup: the jittered-lattice thermal initial condition
  ComponentDescriptor ic;
  ic.name = "thermal_parcelsetup";
  ic.initialisation = [](State& s) {
    if (s.dry_run) return 0;
    if (int rc = ensure_context(s)) return rc;
    const Options& o = s.options;
    pmpic_thermal_params p{};
    p.nx = (int32_t)o.integer("nx");
    p.ny = (int32_t)o.integer("ny");
    p.nz = (int32_t)o.integer("nz");
    p.lx = o.real("xmax") - o.real("xmin");
    p.ly = o.real("ymax") - o.real("ymin");
    p.lz = o.real("zmax") - o.real("zmin");
    p.sub = (int32_t)o.integer("parcels_per_cell_dir", 2);
    p.jitter = o.real("thermal_jitter", 0.25);
    p.seed = (uint64_t)o.integer("thermal_seed", 1);
    p.xc = o.real("thermal_xc", 0.5 * p.lx);
    p.yc = o.real("thermal_yc", 0.5 * p.ly);
    p.zc = o.real("thermal_zc", 0.6);
    p.radius = o.real("thermal_radius", 0.4);
    p.excess = o.real("thermal_excess", 1.0);
    p.h_in = o.real("thermal_humidity", 0.95);
    p.h_env0 = o.real("environment_humidity", 0.3);
    p.z_strat = o.real("stratification_height", 1.2);
    p.n2 = o.real("n2", 1.0);
    int64_t n = pmpic_setup_count(&p);
    if (n <= 0) return (int)PMPIC_ERR_CONFIG;
    std::vector<double> a[11];
    for (auto& x : a) x.resize((size_t)n);
    int rc = pmpic_setup_thermal(&p, n, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(),
                                 a[5].data(), a[6].data(), a[7].data(), a[8].data(), a[9].data(), a[10].data());
    if (rc) return rc;
    return check(s, pmpic_upload_parcels(s.gpu, n, a[0].data(), a[1].data(), a[2].data(), a[3].data(),
                                         a[4].data(), a[5].data(), a[6].data(), a[7].data(), a[8].data(),
                                         a[9].data(), a[10].data()),
                 "pmpic_upload_parcels");
  };
  v.push_back(ic);
  // termination_check (terminationcheck.F90:91-147): time and step limits
  ComponentDescriptor term;
  term.name = "termination_check";
  term.timestep = [](State& s) {
    if (s.dry_run) s.trace.push_back("termination_check");
    // continue while mod(timestep, nn_timesteps) /= 0 (when nn_timesteps > 0)
    // and time < termination_time; the step that sees the stop still runs
    // its remaining groups (timestepper.F90:28-42 calls every group)
    long long nmax = s.options.integer("nn_timesteps", -1);
    s.continue_timestep = !(nmax > 0 && s.timestep % nmax == 0);
    if (s.continue_timestep && s.options.has("termination_time"))
      s.continue_timestep = s.time < s.options.real("termination_time");
    return 0;
  };
  v.push_back(term);
  // model_synopsis: one line of step information every display_synopsis_frequency steps
  ComponentDescriptor syn;
  syn.name = "model_synopsis";
  syn.timestep = [](State& s) {
    if (s.dry_run) {
      s.trace.push_back("model_synopsis");
      return 0;
    }
    long long every = s.options.integer("display_synopsis_frequency", 1);
    if (every > 0 && s.timestep % every == 0)
      std::printf("step %lld time %.6f dt %.6g parcels %lld split %lld removed %lld added %lld limiter %d\n",
                  s.timestep, s.time, s.dtm, (long long)s.info.n_parcels, (long long)s.info.n_split,
                  (long long)s.info.n_removed, (long long)s.info.n_added, s.info.limiter);
    return 0;
  };
  v.push_back(syn);
  return v;
}

// ---- registry + timestepper ---------------------------------------------------------
struct Group {
  std::string name;
  bool rk = false;
  std::vector<const ComponentDescriptor*> members;
};

class Registry {
 public:
  std::vector<ComponentDescriptor> available;
  std::vector<const ComponentDescriptor*> init_order, final_order;
  std::vector<Group> groups;

  const ComponentDescriptor* find(const std::string& n) const {
    for (auto& c : available)
      if (c.name == n) return &c;
    return nullptr;
  }
  bool enabled(const Options& o, const std::string& n) const { return o.logical(n + "_enabled", false); }

  // registry.F90:101-131, :472-510; timestepper groups from group_names /
  // <group>_group_type / <group>_group_contents
  bool build(const Options& o, std::string* err) {
    available = all_components();
    for (const std::string& n : o.list("initialisation_stage_ordering"))
      if (const auto* c = find(n))
        if (enabled(o, n) && c->initialisation) init_order.push_back(c);
    for (const std::string& n : o.list("finalisation_stage_ordering"))
      if (const auto* c = find(n))
        if (enabled(o, n) && c->finalisation) final_order.push_back(c);
    for (const std::string& gname : o.list("group_names")) {
      Group g;
      g.name = gname;
      std::string type = Options::lower(o.str(gname + "_group_type"));
      if (type == "rk_integrated") g.rk = true;
      else if (type != "entire") {
        *err = "group type '" + type + "' of group " + gname + " is not supported";
        return false;
      }
      for (const std::string& n : o.list(gname + "_group_contents"))
        if (const auto* c = find(n))
          if (enabled(o, n) && c->timestep) g.members.push_back(c);
      groups.push_back(g);
    }
    return true;
  }
};

// timestepper.F90:29-106 and monc.F90:200-235
static int run(State& s, Registry& reg) {
  for (const auto* c : reg.init_order) {
    int rc = c->initialisation(s);
    if (rc) {
      release_context(s);
      return rc;
    }
  }
  if (s.rksteps <= 0) {
    std::fprintf(stderr, "Error: number of integrator steps has not been defined.\n");  // timestepper.F90:95-98
    return PMPIC_ERR_CONFIG;
  }
  int rc = 0;
  s.timestep = 1;  // state.F90:54
  while (s.continue_timestep && rc == 0) {
    for (const Group& g : reg.groups) {
      int reps = g.rk ? s.rksteps : 1;
      for (int r = 0; r < reps && rc == 0; ++r)
        for (const auto* c : g.members) {
          rc = c->timestep(s);
          if (rc) break;
        }
      if (rc) break;
    }
    if (s.dry_run) s.continue_timestep = false;  // one step's callback order
    if (s.continue_timestep) {
      s.timestep += 1;
      s.time += s.dtm;
      s.iterations += 1;
    }
  }
  for (const auto* c : reg.final_order) c->finalisation(s);
  release_context(s);
  return rc;
}

}  // namespace monc

int main(int argc, char** argv) {
  monc::State s;
  std::string config, err;
  std::vector<std::string> overrides;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a.rfind("--config=", 0) == 0) config = a.substr(9);
    else if (a == "--dry-run") s.dry_run = true;
    else if (a.rfind("--", 0) == 0) overrides.push_back(a.substr(2));
  }
  if (config.empty()) {
    std::fprintf(stderr, "usage: pmpic_monc --config=FILE [--key=value ...] [--dry-run]\n");
    return 2;
  }
  // command-line options are loaded before and after the file (monc.F90:116-136)
  for (auto& o : overrides) s.options.apply_line(o, "", 0, &err);
  if (!s.options.load(config, 0, &err)) {
    std::fprintf(stderr, "%s\n", err.c_str());
    return 2;
  }
  for (auto& o : overrides) s.options.apply_line(o, "", 0, &err);
  monc::Registry reg;
  if (!reg.build(s.options, &err)) {
    std::fprintf(stderr, "%s\n", err.c_str());
    return 2;
  }
  int rc = monc::run(s, reg);
  if (s.dry_run) {
    std::printf("init:");
    for (const auto* c : reg.init_order) std::printf(" %s", c->name.c_str());
    std::printf("\nstep:");
    for (auto& n : s.trace) std::printf(" %s", n.c_str());
    std::printf("\n");
  }
  return rc == 0 ? 0 : 1;
}
