// C ABI: error reporting, configuration (MPI_3DCompact.in reader), the
// derivative / filter operator objects and host utilities.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

#include "mc3d_internal.h"

namespace mc3d {
static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }
int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
}  // namespace mc3d

using namespace mc3d;

struct mc3d_op_s {
    LineOpHost host;
    LineOpBuf buf;
    int dir = 0;
    Grid3 g{};
    int bc_types[3] = {0, 0, 0};
    bool filter = false;
    int precision = MC3D_FP64;
    int device = 0;
    // TPB form of a periodic derivative: the scheme, the same left-hand side
    // with an identity right-hand-side stencil, and one field of scratch for
    // the right-hand side (both made at the first TPB call)
    int fd_type = -1;
    double dh = 1.0;
    LineOpBuf tpb_solve;
    bool tpb_ready = false;
    void *tpb_rhs = nullptr;
};

extern "C" {

const char *mc3d_last_error(void) { return g_last_error.c_str(); }

int mc3d_config_default(mc3d_config *c) {
    if (!c) return fail(MC3D_ERR_ARG, "null config");
    std::memset(c, 0, sizeof(*c));
    // defaults of Options (src/Options.hpp:226-428)
    c->Nx = c->Ny = c->Nz = 0;
    for (int d = 0; d < 3; d++) {
        c->bc_type[d] = MC3D_PERIODIC_SOLVE;
        c->fd_type[d] = MC3D_PADE6;
    }
    for (int f = 0; f < 6; f++) c->bc_kind[f] = MC3D_BC_PERIODIC;
    c->filter_type = MC3D_COMPACT10;
    c->alphaF = 0.45;
    c->mu_ref = 0.0;
    c->rk_type = MC3D_RK4;
    c->ts_type = MC3D_CONST_CFL;
    c->cfl = 0.5;
    c->dt = -1.0;
    c->filter_step = 1;
    c->substep_filtering = 0;
    c->max_time_step = 10000;
    c->max_time = 1000.0;
    c->les_model = MC3D_NOMODEL;
    c->les_averaging = MC3D_AVG_NONE;
    c->time_step0 = 0;
    c->time0 = 0.0;
    c->precision = MC3D_FP64;
    c->reference_quirks = 1;
    c->dsm_test_filter = 1;   // src/Options.hpp:424-425 defaults
    c->dsm_use_taukk = 1;
    c->sponge_kind = MC3D_SPONGE_RECTILINEAR;
    c->sponge_strength = 1.0;   // src/Options.hpp:323
    for (int f = 0; f < 6; f++) c->sponge_rect_perc[f] = 0.0;
    c->sponge_cyl_orient = 2;
    for (int d = 0; d < 3; d++) c->sponge_cyl_axis[d] = 0.0;
    c->sponge_rmin = 0.0;
    for (int f = 0; f < 6; f++) c->wall_velocity[f][0] = c->wall_velocity[f][1] = 0.0;
    c->mlp_fallback_frac = 1e-3;
    for (int d = 0; d < 3; d++)
        for (int e = 0; e < 3; e++) c->periodic_disp[d][e] = 0.0;
    c->dump_step = 1000;   // src/Options.hpp:237
    c->from_restart = c->only_grid_from_restart = c->sponge_avg_from_restart = 0;
    c->restart_file[0] = c->sponge_avg_file[0] = '\0';
    c->velocity_stats = c->thermo_stats = 0;
    c->stats_interval = 5;   // src/Options.hpp:417
    c->sponge_avg_time = 1.0;       // src/Options.hpp:321
    c->sponge_p_inf = 1.0 / 1.4;    // src/Options.hpp:322
    c->sponge_relax = 0;
    c->lean_storage = 0;
    c->lean_slab = 0;
    c->stats_avg_type = MC3D_AVG_NONE;
    c->velocity_stats_from_restart = c->thermo_stats_from_restart = 0;
    c->velocity_stats_file[0] = c->thermo_stats_file[0] = '\0';
    return MC3D_OK;
}

}  // extern "C"

namespace {

std::string trim(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

struct Ini {
    std::map<std::string, std::string> kv;
    bool has(const std::string &k) const { return kv.count(k) != 0; }
    const std::string &get(const std::string &k) const { return kv.at(k); }
};

// every key Options registers (src/Options.hpp:133-206) plus the [GPU] keys
const char *KNOWN_KEYS[] = {
    "TIMESTEPPING.TSTYPE", "TIMESTEPPING.CFL", "TIMESTEPPING.DT", "TIMESTEPPING.MAXTIME",
    "TIMESTEPPING.MAXTIMESTEP", "TIMESTEPPING.FILTERSTEP", "TIMESTEPPING.SUBSTEPFILTERING",
    "TIMESTEPPING.CHECKSTEP", "TIMESTEPPING.DUMPSTEP", "BC.BCXTYPE", "BC.BCYTYPE", "BC.BCZTYPE", "BC.BCX0",
    "BC.BCX1", "BC.BCY0", "BC.BCY1", "BC.BCZ0", "BC.BCZ1", "BC.PERIODICDISPX_X", "BC.PERIODICDISPX_Y",
    "BC.PERIODICDISPX_Z", "BC.PERIODICDISPY_X", "BC.PERIODICDISPY_Y", "BC.PERIODICDISPY_Z",
    "BC.PERIODICDISPZ_X", "BC.PERIODICDISPZ_Y", "BC.PERIODICDISPZ_Z", "SPONGE.KIND", "SPONGE.AVGTIME",
    "SPONGE.PINF", "SPONGE.STRENGTH", "SPONGE.RECTX0PERC", "SPONGE.RECTY0PERC", "SPONGE.RECTZ0PERC",
    "SPONGE.RECTX1PERC", "SPONGE.RECTY1PERC", "SPONGE.RECTZ1PERC", "SPONGE.CYLAXIS_ORIENT", "SPONGE.CYLAXIS_X",
    "SPONGE.CYLAXIS_Y", "SPONGE.CYLAXIS_Z", "SPONGE.RMIN", "DOMAIN.NX", "DOMAIN.NY", "DOMAIN.NZ",
    "PENCILDECOMP.PROW", "PENCILDECOMP.PCOL", "SOLVER.ALPHAF", "SOLVER.MU_REF", "SOLVER.USETIMING",
    "SOLVER.XFDTYPE", "SOLVER.YFDTYPE", "SOLVER.ZFDTYPE", "SOLVER.FILTERTYPE", "SOLVER.RKTYPE",
    "RESTART.FROMRESTART", "RESTART.ONLYGRIDFROMRESTART", "RESTART.FILENAME", "RESTART.SPONGEAVGFROMRESTART",
    "RESTART.SPONGEAVGFILENAME", "STATS.VELOCITYSTATS", "STATS.THERMOSTATS", "STATS.VELOCITYSTATSFROMRESTART",
    "STATS.THERMOSTATSFROMRESTART", "STATS.VELOCITYSTATSFILENAME", "STATS.THERMOSTATSFILENAME",
    "STATS.STATSAVGTYPE", "STATS.INTERVAL", "LES.LESMODEL", "LES.LESAVERAGING", "LES.DSMTESTFILTER",
    "LES.DSMUSETAUKK", "LES.DSMCOEFFRANGE", "LES.MLPFALLBACKFRAC", "GPU.PRECISION", "GPU.REFERENCEQUIRKS",
    "GPU.STORAGE", "GPU.LEANSLAB"};

struct CfgError {
    std::string msg;
};

bool parse_bool(const std::string &k, const std::string &v) {
    std::string s = v;
    std::transform(s.begin(), s.end(), s.begin(), ::tolower);
    if (s == "1" || s == "true" || s == "yes" || s == "on") return true;
    if (s == "0" || s == "false" || s == "no" || s == "off") return false;
    throw CfgError{"invalid bool for " + k + ": " + v};
}
double parse_double(const std::string &k, const std::string &v) {
    char *end = nullptr;
    double x = std::strtod(v.c_str(), &end);
    if (end == v.c_str()) throw CfgError{"invalid number for " + k + ": " + v};
    return x;
}
int parse_int(const std::string &k, const std::string &v) {
    char *end = nullptr;
    long x = std::strtol(v.c_str(), &end, 10);
    if (end == v.c_str()) throw CfgError{"invalid integer for " + k + ": " + v};
    return (int)x;
}

int parse_enum(const Ini &ini, const std::string &k, const std::map<std::string, int> &m) {
    if (!ini.has(k)) throw CfgError{k + " not specified"};   // parse*String aborts (Options.cpp)
    auto it = m.find(ini.get(k));
    if (it == m.end()) throw CfgError{"unknown value for " + k + ": " + ini.get(k)};
    return it->second;
}

}  // namespace

extern "C" int mc3d_config_from_ini(const char *path, mc3d_config *c) {
    if (!path || !c) return fail(MC3D_ERR_ARG, "null argument");
    mc3d_config_default(c);
    std::ifstream in(path);
    if (!in) return fail(MC3D_ERR_CONFIG, std::string("cannot open ") + path);
    Ini ini;
    std::string line, prefix;
    try {
        while (std::getline(in, line)) {
            size_t h = line.find('#');
            if (h != std::string::npos) line = line.substr(0, h);
            line = trim(line);
            if (line.empty()) continue;
            if (line[0] == '[') {
                size_t e = line.find(']');
                if (e == std::string::npos) throw CfgError{"bad section header: " + line};
                prefix = trim(line.substr(1, e - 1)) + ".";
                continue;
            }
            size_t eq = line.find('=');
            if (eq == std::string::npos) throw CfgError{"syntax error: " + line};
            std::string k = prefix + trim(line.substr(0, eq));
            bool known = false;
            for (const char *kk : KNOWN_KEYS) known = known || k == kk;
            if (!known) throw CfgError{"unrecognised option '" + k + "'"};
            if (!ini.has(k)) ini.kv[k] = trim(line.substr(eq + 1));
        }
        // [TIMESTEPPING] (Options.hpp:224-238)
        c->ts_type = parse_enum(ini, "TIMESTEPPING.TSTYPE", {{"CONST_DT", MC3D_CONST_DT}, {"CONST_CFL", MC3D_CONST_CFL}});
        if (c->ts_type == MC3D_CONST_DT) {
            if (!ini.has("TIMESTEPPING.DT")) throw CfgError{"DT not specified, NEEDS TO BE SPECIFED"};
            c->dt = parse_double("DT", ini.get("TIMESTEPPING.DT"));
            c->cfl = -1.0;
        } else {
            c->cfl = ini.has("TIMESTEPPING.CFL") ? parse_double("CFL", ini.get("TIMESTEPPING.CFL")) : 0.5;
            c->dt = -1.0;
        }
        if (ini.has("TIMESTEPPING.MAXTIME")) c->max_time = parse_double("MAXTIME", ini.get("TIMESTEPPING.MAXTIME"));
        if (ini.has("TIMESTEPPING.MAXTIMESTEP"))
            c->max_time_step = parse_int("MAXTIMESTEP", ini.get("TIMESTEPPING.MAXTIMESTEP"));
        if (ini.has("TIMESTEPPING.FILTERSTEP"))
            c->filter_step = parse_int("FILTERSTEP", ini.get("TIMESTEPPING.FILTERSTEP"));
        if (ini.has("TIMESTEPPING.DUMPSTEP")) c->dump_step = parse_int("DUMPSTEP", ini.get("TIMESTEPPING.DUMPSTEP"));
        if (c->dump_step <= 0) throw CfgError{"DUMPSTEP must be positive"};
        if (ini.has("TIMESTEPPING.SUBSTEPFILTERING"))
            c->substep_filtering = parse_bool("SUBSTEPFILTERING", ini.get("TIMESTEPPING.SUBSTEPFILTERING"));
        // [DOMAIN] (required unless restarting, Options.hpp:380-385)
        bool restart = ini.has("RESTART.FROMRESTART") && parse_bool("FROMRESTART", ini.get("RESTART.FROMRESTART"));
        bool gridrs = ini.has("RESTART.ONLYGRIDFROMRESTART") &&
                      parse_bool("ONLYGRIDFROMRESTART", ini.get("RESTART.ONLYGRIDFROMRESTART"));
        if (!ini.has("RESTART.FROMRESTART")) throw CfgError{"fromRestart not specified, NEEDS TO BE SPECIFED"};
        if (!ini.has("RESTART.ONLYGRIDFROMRESTART"))
            throw CfgError{"onlyGridFromRestart not specified, NEEDS TO BE SPECIFED"};
        if (!ini.has("RESTART.SPONGEAVGFROMRESTART"))
            throw CfgError{"spongeFromRestart not specified, NEEDS TO BE SPECIFED"};
        if (restart && gridrs) throw CfgError{"'only use grid from restart file' and 'from restart file' conflict"};
        c->from_restart = restart ? 1 : 0;
        c->only_grid_from_restart = gridrs ? 1 : 0;
        if (restart || gridrs) {
            if (!ini.has("RESTART.FILENAME")) throw CfgError{"restart filename not specified, NEEDS TO BE SPECIFED"};
            const std::string fn = ini.get("RESTART.FILENAME");
            if (fn.size() >= sizeof(c->restart_file)) throw CfgError{"RESTART.FILENAME is too long"};
            std::snprintf(c->restart_file, sizeof(c->restart_file), "%s", fn.c_str());
            // grid sizes from the file's header (src/MPI_3DCompact.cpp:80-110)
            if (read_solution_header(c->restart_file, nullptr, nullptr, &c->Nx, &c->Ny, &c->Nz))
                throw CfgError{"ERROR: Couldn't open file " + fn};
        } else {
            const char *dk[3] = {"DOMAIN.NX", "DOMAIN.NY", "DOMAIN.NZ"};
            int *dn[3] = {&c->Nx, &c->Ny, &c->Nz};
            for (int d = 0; d < 3; d++) {
                if (!ini.has(dk[d])) throw CfgError{std::string(dk[d]) + " not specified, NEEDS TO BE SPECIFED"};
                *dn[d] = parse_int(dk[d], ini.get(dk[d]));
            }
        }
        c->sponge_avg_from_restart = parse_bool("SPONGEAVGFROMRESTART", ini.get("RESTART.SPONGEAVGFROMRESTART")) ? 1 : 0;
        if (c->sponge_avg_from_restart) {
            if (!ini.has("RESTART.SPONGEAVGFILENAME"))
                throw CfgError{"sponge_filename not specified, NEEDS TO BE SPECIFED"};
            const std::string fn = ini.get("RESTART.SPONGEAVGFILENAME");
            if (fn.size() >= sizeof(c->sponge_avg_file)) throw CfgError{"RESTART.SPONGEAVGFILENAME is too long"};
            std::snprintf(c->sponge_avg_file, sizeof(c->sponge_avg_file), "%s", fn.c_str());
        }
        if (c->Nx <= 10 || c->Ny <= 10 || c->Nz <= 10)
            throw CfgError{"Number of grid points in any direction must be greater than 10!"};
        // [SOLVER]
        if (ini.has("SOLVER.ALPHAF")) c->alphaF = parse_double("ALPHAF", ini.get("SOLVER.ALPHAF"));
        if (!ini.has("SOLVER.MU_REF")) throw CfgError{"mu_ref not specified, NEEDS TO BE SPECIFED"};
        c->mu_ref = parse_double("MU_REF", ini.get("SOLVER.MU_REF"));
        std::map<std::string, int> fd = {{"CD2", MC3D_CD2}, {"PADE6", MC3D_PADE6}, {"PENTA10", MC3D_PENTA10}};
        c->fd_type[0] = parse_enum(ini, "SOLVER.XFDTYPE", fd);
        c->fd_type[1] = parse_enum(ini, "SOLVER.YFDTYPE", fd);
        c->fd_type[2] = parse_enum(ini, "SOLVER.ZFDTYPE", fd);
        c->filter_type = parse_enum(ini, "SOLVER.FILTERTYPE", {{"COMPACT8", MC3D_COMPACT8}, {"COMPACT10", MC3D_COMPACT10}});
        c->rk_type = parse_enum(ini, "SOLVER.RKTYPE", {{"TVDRK3", MC3D_TVDRK3}, {"RK4", MC3D_RK4},
                                                       {"KENRK4", MC3D_KENRK4}, {"LSLDDRK4", MC3D_LSLDDRK4}});
        // [BC] (Options.hpp:258-318, Options.cpp:175-296)
        std::map<std::string, int> bct = {{"PERIODIC_SOLVE", MC3D_PERIODIC_SOLVE}, {"DIRICHLET_SOLVE", MC3D_DIRICHLET_SOLVE}};
        std::map<std::string, int> bck = {{"INTERNALLY_PERIODIC", MC3D_BC_INTERNALLY_PERIODIC},
                                          {"PERIODIC", MC3D_BC_PERIODIC},
                                          {"ADIABATIC_WALL", MC3D_BC_ADIABATIC_WALL},
                                          {"SPONGE", MC3D_BC_SPONGE},
                                          {"CONST_T_WALL", MC3D_BC_CONST_T_WALL},
                                          {"MOVING_ADIABATIC_WALL", MC3D_BC_MOVING_ADIABATIC_WALL},
                                          {"INLET", MC3D_BC_INLET}};
        const char *ax = "XYZ";
        for (int d = 0; d < 3; d++) c->bc_type[d] = parse_enum(ini, std::string("BC.BC") + ax[d] + "TYPE", bct);
        for (int d = 0; d < 3; d++)
            for (int e = 0; e < 2; e++)
                c->bc_kind[2 * d + e] = parse_enum(ini, std::string("BC.BC") + ax[d] + (char)('0' + e), bck);
        for (int d = 0; d < 3; d++) {
            int k0 = c->bc_kind[2 * d], k1 = c->bc_kind[2 * d + 1];
            bool p0 = k0 == MC3D_BC_PERIODIC, p1 = k1 == MC3D_BC_PERIODIC;
            if (p0 != p1) throw CfgError{std::string(" BC Mismatch for ") + ax[d] + "0-" + ax[d] + "1 Faces! "};
            if (p0)
                for (int e = 0; e < 3; e++) {
                    std::string k = std::string("BC.PERIODICDISP") + ax[d] + "_" + ax[e];
                    if (!ini.has(k)) throw CfgError{k + " not specified, NEEDS TO BE SPECIFED"};
                    c->periodic_disp[d][e] = parse_double(k.c_str() + 3, ini.get(k));
                }
            bool ip0 = p0 || k0 == MC3D_BC_INTERNALLY_PERIODIC, ip1 = p1 || k1 == MC3D_BC_INTERNALLY_PERIODIC;
            if (c->bc_type[d] == MC3D_PERIODIC_SOLVE) {
                if (!ip0 || !ip1) throw CfgError{std::string("PERIODIC_SOLVE in ") + ax[d] + " needs PERIODIC or INTERNALLY_PERIODIC faces"};
                if (p0 != p1) throw CfgError{std::string("mismatched periodic conditions in ") + ax[d]};
            } else if (ip0 || ip1) {
                throw CfgError{std::string("DIRICHLET_SOLVE in ") + ax[d] + " cannot have periodic faces"};
            }
        }
        // [STATS], [LES]
        c->stats_avg_type = parse_enum(ini, "STATS.STATSAVGTYPE",
                                       {{"NONE", MC3D_AVG_NONE}, {"XI1_AVG", MC3D_AVG_XI1}, {"XI2_AVG", MC3D_AVG_XI2},
                                        {"XI3_AVG", MC3D_AVG_XI3}, {"LOCAL", MC3D_AVG_LOCAL}, {"GLOBAL", MC3D_AVG_GLOBAL}});
        if (ini.has("STATS.VELOCITYSTATS")) c->velocity_stats = parse_bool("VELOCITYSTATS", ini.get("STATS.VELOCITYSTATS"));
        if (ini.has("STATS.THERMOSTATS")) c->thermo_stats = parse_bool("THERMOSTATS", ini.get("STATS.THERMOSTATS"));
        if (ini.has("STATS.INTERVAL")) c->stats_interval = parse_int("INTERVAL", ini.get("STATS.INTERVAL"));
        if (c->stats_interval <= 0) throw CfgError{"STATS.INTERVAL must be positive"};
        {
            const char *flag[2] = {"STATS.VELOCITYSTATSFROMRESTART", "STATS.THERMOSTATSFROMRESTART"};
            const char *file[2] = {"STATS.VELOCITYSTATSFILENAME", "STATS.THERMOSTATSFILENAME"};
            const char *what[2] = {"velocityStatsFromRestart", "thermoStatsFromRestart"};
            int on[2] = {c->velocity_stats, c->thermo_stats};
            int *from[2] = {&c->velocity_stats_from_restart, &c->thermo_stats_from_restart};
            char *dst[2] = {c->velocity_stats_file, c->thermo_stats_file};
            for (int k = 0; k < 2; k++) {
                if (!on[k]) continue;
                if (!ini.has(flag[k])) throw CfgError{std::string(what[k]) + " not specified, NEEDS TO BE SPECIFED"};
                *from[k] = parse_bool(flag[k], ini.get(flag[k])) ? 1 : 0;
                if (*from[k]) {
                    if (!ini.has(file[k])) throw CfgError{std::string(file[k]) + " not specified, NEEDS TO BE SPECIFED"};
                    const std::string fn = ini.get(file[k]);
                    if (fn.size() >= 512) throw CfgError{std::string(file[k]) + " is too long"};
                    std::snprintf(dst[k], 512, "%s", fn.c_str());
                }
            }
        }
        c->les_model = parse_enum(ini, "LES.LESMODEL", {{"NOMODEL", MC3D_NOMODEL}, {"NONE", MC3D_NOMODEL},
                                                        {"VREMAN", MC3D_VREMAN}, {"DSM", MC3D_DSM},
                                                        {"MLP", MC3D_MLPSGS}});
        c->les_averaging = parse_enum(ini, "LES.LESAVERAGING",
                                      {{"NONE", MC3D_AVG_NONE}, {"XI1_AVG", MC3D_AVG_XI1}, {"XI2_AVG", MC3D_AVG_XI2},
                                       {"XI3_AVG", MC3D_AVG_XI3}, {"LOCAL", MC3D_AVG_LOCAL}, {"GLOBAL", MC3D_AVG_GLOBAL}});
        if (ini.has("LES.DSMTESTFILTER")) {
            c->dsm_test_filter = parse_int("DSMTESTFILTER", ini.get("LES.DSMTESTFILTER"));
            // DSMSGS aborts on any other value (src/DSMSGS.hpp:57-67)
            if (c->dsm_test_filter != 1 && c->dsm_test_filter != 2) throw CfgError{"DSMTESTFILTER must be 1 or 2"};
        }
        if (ini.has("LES.DSMUSETAUKK")) c->dsm_use_taukk = parse_bool("DSMUSETAUKK", ini.get("LES.DSMUSETAUKK"));
        if (ini.has("LES.MLPFALLBACKFRAC")) {
            c->mlp_fallback_frac = parse_double("MLPFALLBACKFRAC", ini.get("LES.MLPFALLBACKFRAC"));
            if (!(c->mlp_fallback_frac >= 0.0 && c->mlp_fallback_frac <= 1.0))
                throw CfgError{"MLPFALLBACKFRAC must lie in [0, 1]"};
        }
        // [SPONGE]: read when a face is a sponge (src/Options.hpp:314-358)
        bool sponge = false;
        for (int f = 0; f < 6; f++) sponge = sponge || c->bc_kind[f] == MC3D_BC_SPONGE;
        if (sponge) {
            c->sponge_kind = parse_enum(ini, "SPONGE.KIND", {{"RECTILINEAR", MC3D_SPONGE_RECTILINEAR},
                                                             {"CYLINDRICAL", MC3D_SPONGE_CYLINDRICAL}});
            if (ini.has("SPONGE.STRENGTH")) c->sponge_strength = parse_double("STRENGTH", ini.get("SPONGE.STRENGTH"));
            if (ini.has("SPONGE.AVGTIME")) c->sponge_avg_time = parse_double("AVGTIME", ini.get("SPONGE.AVGTIME"));
            if (ini.has("SPONGE.PINF")) c->sponge_p_inf = parse_double("PINF", ini.get("SPONGE.PINF"));
            const char *pk[6] = {"SPONGE.RECTX0PERC", "SPONGE.RECTX1PERC", "SPONGE.RECTY0PERC",
                                 "SPONGE.RECTY1PERC", "SPONGE.RECTZ0PERC", "SPONGE.RECTZ1PERC"};
            if (c->sponge_kind == MC3D_SPONGE_RECTILINEAR) {
                for (int f = 0; f < 6; f++)
                    if (c->bc_kind[f] == MC3D_BC_SPONGE) {
                        if (!ini.has(pk[f])) throw CfgError{std::string(pk[f]) + " is required"};
                        c->sponge_rect_perc[f] = parse_double(pk[f], ini.get(pk[f]));
                    }
            } else {
                const char *ck[4] = {"SPONGE.CYLAXIS_X", "SPONGE.CYLAXIS_Y", "SPONGE.CYLAXIS_Z", "SPONGE.RMIN"};
                if (!ini.has("SPONGE.CYLAXIS_ORIENT")) throw CfgError{"SPONGE.CYLAXIS_ORIENT is required"};
                c->sponge_cyl_orient = parse_int("CYLAXIS_ORIENT", ini.get("SPONGE.CYLAXIS_ORIENT"));
                if (c->sponge_cyl_orient < 0 || c->sponge_cyl_orient > 2)
                    throw CfgError{"SPONGE.CYLAXIS_ORIENT must be 0, 1 or 2"};
                for (int k = 0; k < 4; k++) {
                    if (!ini.has(ck[k])) throw CfgError{std::string(ck[k]) + " is required"};
                    double v = parse_double(ck[k], ini.get(ck[k]));
                    if (k < 3) c->sponge_cyl_axis[k] = v;
                    else c->sponge_rmin = v;
                }
            }
        }
        // [GPU]
        if (ini.has("GPU.PRECISION"))
            c->precision = parse_enum(ini, "GPU.PRECISION", {{"FP64", MC3D_FP64}, {"FP32BULK", MC3D_FP32BULK}});
        if (ini.has("GPU.STORAGE")) c->lean_storage = parse_enum(ini, "GPU.STORAGE", {{"FULL", 0}, {"LEAN", 1}});
        if (ini.has("GPU.LEANSLAB")) c->lean_slab = std::stoi(ini.get("GPU.LEANSLAB"));
        if (ini.has("GPU.REFERENCEQUIRKS"))
            c->reference_quirks = parse_bool("REFERENCEQUIRKS", ini.get("GPU.REFERENCEQUIRKS"));
    } catch (const CfgError &e) {
        return fail(MC3D_ERR_CONFIG, e.msg);
    }
    return MC3D_OK;
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
static int op_finish(mc3d_op o, mc3d_op *out) {
    int rc = upload_line_op(o->host, o->precision, o->buf);
    if (rc) {
        delete o;
        return rc;
    }
    *out = o;
    return MC3D_OK;
}

extern "C" int mc3d_deriv_create(int fd_type, int bc_type, int dir, int Nx, int Ny, int Nz, double dh, int precision,
                                 int device, mc3d_op *out) {
    if (!out) return fail(MC3D_ERR_ARG, "null argument");
    *out = nullptr;
    if (dir < 0 || dir > 2) return fail(MC3D_ERR_ARG, "dir must be 0, 1 or 2");
    if (precision != MC3D_FP64 && precision != MC3D_FP32BULK) return fail(MC3D_ERR_ARG, "bad precision");
    if (!(dh > 0)) return fail(MC3D_ERR_ARG, "dh must be positive");
    MC3D_CUDA_TRY(cudaSetDevice(device));
    mc3d_op o = new mc3d_op_s();
    o->dir = dir;
    o->g = Grid3{Nx, Ny, Nz};
    for (int d = 0; d < 3; d++) o->bc_types[d] = MC3D_PERIODIC_SOLVE;
    o->bc_types[dir] = bc_type;
    o->precision = precision;
    o->device = device;
    o->fd_type = fd_type;
    o->dh = dh;
    int N[3] = {Nx, Ny, Nz};
    try {
        o->host = build_deriv_op(fd_type, bc_type, N[dir], dh);
    } catch (const std::exception &e) {
        delete o;
        return fail(MC3D_ERR_CONFIG, e.what());
    }
    return op_finish(o, out);
}

extern "C" int mc3d_filter_create(int filter_type, double alphaF, int dir, const int bc_types[3], int Nx, int Ny,
                                  int Nz, int precision, int device, mc3d_op *out) {
    if (!out || !bc_types) return fail(MC3D_ERR_ARG, "null argument");
    *out = nullptr;
    if (dir < 0 || dir > 2) return fail(MC3D_ERR_ARG, "dir must be 0, 1 or 2");
    if (precision != MC3D_FP64 && precision != MC3D_FP32BULK) return fail(MC3D_ERR_ARG, "bad precision");
    MC3D_CUDA_TRY(cudaSetDevice(device));
    mc3d_op o = new mc3d_op_s();
    o->dir = dir;
    o->g = Grid3{Nx, Ny, Nz};
    for (int d = 0; d < 3; d++) o->bc_types[d] = bc_types[d];
    o->filter = true;
    o->precision = precision;
    o->device = device;
    int N[3] = {Nx, Ny, Nz};
    try {
        if (filter_type == MC3D_TESTFILTER_PADE || filter_type == MC3D_TESTFILTER_EXP)
            o->host = build_testfilter_op(filter_type, bc_types[dir], N[dir]);
        else
            o->host = build_filter_op(filter_type, alphaF, bc_types[dir], N[dir]);
    } catch (const std::exception &e) {
        delete o;
        return fail(MC3D_ERR_CONFIG, e.what());
    }
    return op_finish(o, out);
}

template <typename R>
static int op_apply_t(mc3d_op o, const void *const *in, void *const *out, int nf, cudaStream_t st) {
    RhsFinalArgs<R> rf{};
    for (int base = 0; base < nf; base += 16) {
        SweepBatch<R> b{};
        b.nf = std::min(16, nf - base);
        for (int f = 0; f < b.nf; f++) {
            b.in[f] = (const R *)in[base + f];
            b.out[f] = (R *)out[base + f];
            if (!b.in[f] || !b.out[f]) return fail(MC3D_ERR_ARG, "null field pointer");
            if ((const void *)b.in[f] == (const void *)b.out[f]) return fail(MC3D_ERR_ARG, "in and out alias");
        }
        const LineOpDev<R> &d = std::is_same<R, float>::value ? *(const LineOpDev<R> *)&o->buf.f32
                                                                : *(const LineOpDev<R> *)&o->buf.f64;
        int rc = launch_sweep<R>(o->dir, o->g, d, b, EPI_STORE, rf, o->bc_types, o->filter, st);
        if (rc) return rc;
    }
    return MC3D_OK;
}

extern "C" int mc3d_op_apply(mc3d_op o, const void *const *in, void *const *out, int nfields, void *stream) {
    if (!o || !in || !out) return fail(MC3D_ERR_ARG, "null argument");
    if (nfields <= 0) return MC3D_OK;
    MC3D_CUDA_TRY(cudaSetDevice(o->device));
    cudaStream_t st = (cudaStream_t)stream;
    return o->precision == MC3D_FP64 ? op_apply_t<double>(o, in, out, nfields, st)
                                     : op_apply_t<float>(o, in, out, nfields, st);
}

extern "C" int mc3d_op_destroy(mc3d_op o) {
    if (!o) return MC3D_OK;
    cudaSetDevice(o->device);
    free_line_op(o->buf);
    free_line_op(o->tpb_solve);
    if (o->tpb_rhs) cudaFree(o->tpb_rhs);
    delete o;
    return MC3D_OK;
}

// ghost planes per side of the TPB form: the BW5 signature (Pade6, CD2) takes
// Nm2, Nm1, Np1, Np2; the BW7 one (Penta10) Nm3 .. Np3
static int tpb_width(const mc3d_op o) { return o->fd_type == MC3D_PENTA10 ? 3 : 2; }

extern "C" int mc3d_op_tpb_ghosts(mc3d_op o, int *per_side) {
    if (!o || !per_side) return fail(MC3D_ERR_ARG, "null argument");
    if (o->filter || o->fd_type < 0) return fail(MC3D_ERR_CONFIG, "TPB is a form of the derivative operators only");
    *per_side = tpb_width(o);
    return MC3D_OK;
}

template <typename R>
static int op_apply_tpb_t(mc3d_op o, const void *const *in, void *const *out, int nf, const void *const *ghosts,
                          cudaStream_t st) {
    const int G = tpb_width(o);
    TpbPlanes<R> gp{};
    gp.G = G;
    gp.H = o->host.H;
    gp.explicit_cd2 = o->fd_type == MC3D_CD2;
    for (int k = 0; k < 7; k++) gp.st[k] = k <= 2 * o->host.H ? o->host.st[k] : 0.0;
    const LineOpBuf &sb = o->tpb_solve;
    const LineOpDev<R> &sd = std::is_same<R, float>::value ? *(const LineOpDev<R> *)&sb.f32
                                                           : *(const LineOpDev<R> *)&sb.f64;
    RhsFinalArgs<R> rf{};
    for (int f = 0; f < nf; f++) {
        if (!in[f] || !out[f]) return fail(MC3D_ERR_ARG, "null field pointer");
        if (in[f] == out[f]) return fail(MC3D_ERR_ARG, "in and out alias");
        for (int m = 0; m < 2 * G; m++) {
            gp.p[m] = (const R *)ghosts[(size_t)f * 2 * G + m];
            if (!gp.p[m]) return fail(MC3D_ERR_ARG, "null ghost plane");
        }
        int rc;
        if (gp.explicit_cd2)   // explicit: the right-hand side is the derivative
            rc = launch_tpb_planes_rhs<R>(o->g, o->dir, (const R *)in[f], gp, o->dh, (R *)out[f], st);
        else {
            rc = launch_tpb_planes_rhs<R>(o->g, o->dir, (const R *)in[f], gp, o->dh, (R *)o->tpb_rhs, st);
            if (!rc) {
                SweepBatch<R> b{};
                b.nf = 1;
                b.in[0] = (const R *)o->tpb_rhs;
                b.out[0] = (R *)out[f];
                rc = launch_sweep<R>(o->dir, o->g, sd, b, EPI_STORE, rf, o->bc_types, false, st);
            }
        }
        if (rc) return rc;
    }
    return MC3D_OK;
}

extern "C" int mc3d_op_apply_tpb(mc3d_op o, const void *const *in, void *const *out, int nfields,
                                 const void *const *ghosts, void *stream) {
    if (!o || !in || !out || !ghosts) return fail(MC3D_ERR_ARG, "null argument");
    if (o->filter || o->fd_type < 0) return fail(MC3D_ERR_CONFIG, "TPB is a form of the derivative operators only");
    if (o->bc_types[o->dir] != MC3D_PERIODIC_SOLVE)
        return fail(MC3D_ERR_CONFIG, "CANT USE calc1stDeriv_TPB for non-periodic boundary conditions!!");
    if (nfields <= 0) return MC3D_OK;
    MC3D_CUDA_TRY(cudaSetDevice(o->device));
    cudaStream_t st = (cudaStream_t)stream;
    if (!o->tpb_ready) {
        if (o->fd_type != MC3D_CD2) {
            LineOpHost sv = o->host;
            for (double &v : sv.st) v = 0.0;
            sv.st[sv.H] = 1.0;
            sv.deriv = false;
            sv.inv_dh = 1.0;
            if (int rc = upload_line_op(sv, o->precision, o->tpb_solve)) return rc;
            const size_t bytes = (size_t)o->g.n() * (o->precision == MC3D_FP64 ? 8 : 4);
            MC3D_CUDA_TRY(cudaMalloc(&o->tpb_rhs, bytes));
        }
        o->tpb_ready = true;
    }
    return o->precision == MC3D_FP64 ? op_apply_tpb_t<double>(o, in, out, nfields, ghosts, st)
                                     : op_apply_tpb_t<float>(o, in, out, nfields, ghosts, st);
}

extern "C" double mc3d_calc_neumann(int fd_type, const double *f) {
    if (!f) return NAN;
    if (fd_type == MC3D_CD2) return (f[0] * 4.0 - f[1] * 1.0) / 3.0;   // src/CD2.cpp:183
    // Pade6 / Penta10 (src/Pade6.cpp:395-397, src/Penta10.cpp:284-286)
    return (f[0] * 360.0 - f[1] * 450.0 + f[2] * 400.0 - f[3] * 225.0 + f[4] * 72.0 - f[5] * 10.0) / 147.0;
}

// ---------------------------------------------------------------------------
// HIT initial-condition generator: the combined LCG + 97-entry shuffle table of
// tests/hit/generate_init_hit.f90:54-81 (randvec)
// ---------------------------------------------------------------------------
extern "C" int mc3d_hit_randvec(int *state, double *r, long long n, double *out) {
    if (!state || !r || !out) return fail(MC3D_ERR_ARG, "null argument");
    const long long m1 = 259200, ia1 = 7141, ic1 = 54773;
    const long long m2 = 134456, ia2 = 8121, ic2 = 28441;
    const long long m3 = 243000, ia3 = 4561, ic3 = 51349;
    const double rm1 = 1.0 / m1, rm2 = 1.0 / m2;
    long long ix1 = state[0], ix2 = state[1], ix3 = state[2];
    for (long long m = 0; m < n; m++) {
        ix1 = (ia1 * ix1 + ic1) % m1;
        ix2 = (ia2 * ix2 + ic2) % m2;
        ix3 = (ia3 * ix3 + ic3) % m3;
        long long j = ((97 * ix3) / m3) % 97;
        out[m] = r[j];
        double v = ((double)ix1 + (double)ix2 * rm2) * rm1;
        r[j] = v > 1.0 ? 1.0 : (v < 0.0 ? 0.0 : v);
    }
    state[0] = (int)ix1;
    state[1] = (int)ix2;
    state[2] = (int)ix3;
    return MC3D_OK;
}
