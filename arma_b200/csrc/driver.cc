// The reference's programme layer on top of the device kernels: the `.arma`
// configuration grammar, the model / velocity-solver registry, the
// generate -> velocity -> write pipeline and the output writers.
//
// Reference: ARMA_driver<T> (src/arma_driver.hh:43-150, src/arma_driver.cc:
// 29-178), sys::parameter_map (src/params.cc:30-57), Grid / Domain / interval
// / Output_flags parsers (src/grid.hh:181-193, src/domain.hh:195-217,
// src/apmath/closed_interval.cc:14-27, src/output_flags.cc:53-87), the AR
// model keys (src/generator/ar_model.cc:156-175,
// src/generator/basic_arma_model.cc:15-31), the ACF wrapper keys
// (src/bits/acf_wrapper.cc:41-70), the NIT keys
// (src/nonlinear/nit_transform.cc:255-278) and the velocity solver keys
// (src/velocity/basic_solver.cc:21-36).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <istream>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

[[noreturn]] void bad(const std::string& name, const std::string& what) {
	throw Error{ARMA_EINVAL, "Bad \"" + name + "\": " + what};
}

// ------------------------------------------------------------- lexing helpers
// Skips blank space and '#' comments (a '#' comments out the rest of its
// line) up to the next token, which stays unread.
std::istream& skip_comments(std::istream& in) {
	for (;;) {
		in >> std::ws;
		if (in.peek() != '#') return in;
		std::string rest;
		std::getline(in, rest);
	}
}

bool expect(std::istream& in, char c) {
	char ch = 0;
	if (in >> std::ws >> ch && ch == c) return true;
	if (in) in.putback(ch);
	in.clear();
	return false;
}

template <class T, int N>
void read_tuple(std::istream& in, T* v, const std::string& name) {
	if (!expect(in, '(')) bad(name, "expecting \"(\"");
	for (int i = 0; i < N; ++i) {
		if (i > 0 && !expect(in, ',')) bad(name, "expecting \",\"");
		if (!(in >> v[i])) bad(name, "expecting a number");
	}
	if (!expect(in, ')')) bad(name, "expecting \")\"");
}

std::string read_word(std::istream& in) {
	std::string w;
	in >> std::ws;
	while (in) {
		const int c = in.peek();
		if (c == EOF || std::isspace(c) || c == '{' || c == '}' || c == ',' || c == '=') break;
		w.push_back(char(in.get()));
	}
	return w;
}

// A parameter map: optional braces, key = value lines, '#' comments, unknown
// keys are an error (the reference sets failbit and reports them).
using Reader = std::function<void(std::istream&, const std::string&)>;

void read_params(std::istream& in, const std::map<std::string, Reader>& params, bool parens,
                 const std::string& where) {
	if (parens && !expect(in, '{')) bad(where, "expecting \"{\"");
	std::string name;
	while (in >> skip_comments) {
		if (parens && expect(in, '}')) return;
		in >> std::ws;
		if (!std::getline(in, name, '=')) break;
		while (!name.empty() && name.back() <= ' ') name.pop_back();
		auto it = params.find(name);
		if (it == params.end()) throw Error{ARMA_EINVAL, "Unknown parameter: \"" + name + "\"."};
		it->second(in, name);
	}
	if (parens) bad(where, "expecting \"}\"");
}

template <class T>
Reader number(T* v) {
	return [v](std::istream& in, const std::string& n) {
		if (!(in >> *v)) bad(n, "expecting a number");
	};
}

// depth accepts "inf" (infinite depth, an extension)
Reader real_or_inf(double* v) {
	return [v](std::istream& in, const std::string& n) {
		std::string w = read_word(in);
		if (w == "inf" || w == "infinity") {
			*v = std::numeric_limits<double>::infinity();
			return;
		}
		char* end = nullptr;
		*v = std::strtod(w.c_str(), &end);
		if (w.empty() || *end) bad(n, w);
	};
}

template <class T, int N>
Reader tuple(T* v) {
	return [v](std::istream& in, const std::string& n) { read_tuple<T, N>(in, v, n); };
}

}  // namespace

// ------------------------------------------------------------- configuration
struct Grid3 {
	int n[3] = {0, 0, 0};
	double len[3] = {0, 0, 0};
	double delta(int i) const { return len[i] / std::max(n[i] - 1, 1); }
};

// Grid: "(n,n,n)" or "(n,n,n) : (L,L,L)"; without lengths the patch size is 1.
void read_grid(std::istream& in, Grid3* g, const std::string& name) {
	read_tuple<int, 3>(in, g->n, name);
	if (expect(in, ':')) {
		read_tuple<double, 3>(in, g->len, name);
	} else {
		for (int i = 0; i < 3; ++i) g->len[i] = g->n[i] - 1;
	}
	for (int i = 0; i < 3; ++i)
		if (g->n[i] <= 0 || !(g->len[i] > 0.0) || !std::isfinite(g->len[i])) bad(name, "non-positive");
}

struct Domain2 {
	double lo[2] = {0, 0}, hi[2] = {0, 0};
	int n[2] = {1, 1};
	double at(int i, int dim) const {
		const int np = std::max(n[dim] - 1, 1);
		return lo[dim] + (hi[dim] - lo[dim]) / np * i;
	}
};

// Domain: "from (a,b) to (c,d) npoints (n,m)" in any order.
void read_domain(std::istream& in, Domain2* d, const std::string& name) {
	*d = Domain2();
	for (int k = 0; k < 3; ++k) {
		const std::string p = read_word(in);
		if (p == "from") read_tuple<double, 2>(in, d->lo, name);
		else if (p == "to") read_tuple<double, 2>(in, d->hi, name);
		else if (p == "npoints") read_tuple<int, 2>(in, d->n, name);
		else bad(name, "bad prefix: " + p);
	}
	if (d->n[0] <= 0 || d->n[1] <= 0) bad(name, "npoints");
	for (int i = 0; i < 2; ++i)
		if (!std::isfinite(d->lo[i]) || !std::isfinite(d->hi[i])) bad(name, "not finite");
}

void read_interval(std::istream& in, double* ab, const std::string& name) {
	if (!expect(in, '[')) bad(name, "expecting \"[\"");
	in >> ab[0];
	if (!expect(in, ',')) bad(name, "expecting \",\"");
	in >> ab[1];
	if (!expect(in, ']')) bad(name, "expecting \"]\"");
	if (!(ab[0] <= ab[1])) bad(name, "empty interval");
}

// Output flags (src/output_flags.cc:13-23, 53-87): comma-separated names up to
// the end of the line; "none" clears; "surface" alone implies "blitz".
enum Flag { F_NONE, F_SUMMARY, F_QQ, F_WAVES, F_ACF, F_CSV, F_BLITZ, F_BINARY, F_SURFACE };
const char* kFlagNames[] = {"none", "summary", "qq",    "waves",  "acf",
                            "csv",  "blitz",   "binary", "surface"};

unsigned read_flags(std::istream& in, const std::string& key) {
	unsigned flags = 0;
	std::string name;
	bool stopped = false;
	while (!stopped && !in.eof()) {
		const int ch = in.get();
		if (ch == '\n') stopped = true;
		if (ch == '\n' || ch == ',' || ch == EOF) {
			int f = -1;
			for (int k = 0; k < 9; ++k)
				if (name == kFlagNames[k]) f = k;
			if (f < 0) throw Error{ARMA_EINVAL, "Invalid output flag: " + name};
			if (f == F_NONE) flags = 0;
			else flags |= 1u << f;
			name.clear();
		} else if (!std::isspace(ch)) {
			name.push_back(char(ch));
		}
	}
	in.clear();
	if ((flags & (1u << F_SURFACE)) &&
	    !(flags & ((1u << F_BLITZ) | (1u << F_CSV) | (1u << F_BINARY))))
		flags |= 1u << F_BLITZ;
	(void)key;
	return flags;
}

struct ArConfig {
	bool ma = false;  // model = MA (else AR)
	Grid3 out_grid;
	bool no_seed = false;
	bool has_seed = false;
	uint32_t seed = 0;
	bool nit = false;
	int nit_dist = ARMA_NIT_GRAM_CHARLIER;
	double nit_params[3] = {0, 3, 0};
	double cdf_interval[2] = {0, 1};
	double cdf_eps = 1e-6;
	int cdf_iter = 100;
	int acf_kind = -1;      // analytic ACF (with `grid`)
	Grid3 acf_grid;
	bool acf_empirical = false;  // wave-group ACF (without `grid`)
	EmpiricalAcf wave;
	double amplitude = 1, velocity = 0, alpha[3] = {0, 0, 0}, beta[2] = {0, 0};
	unsigned output = 0;
	int order[3] = {0, 0, 0};
	bool validate = true;
	std::string algorithm = "choi_recursive";
	int partition[3] = {0, 0, 0};
	int precision = ARMA_FP64;
	std::string mt_file = "mt.dat";
};

void read_bisection(std::istream& in, double* ab, double* eps, int* iter, const std::string& n) {
	std::map<std::string, Reader> p = {
	    {"interval", [ab](std::istream& s, const std::string& k) { read_interval(s, ab, k); }},
	    {"absolute_error", number(eps)},
	    {"max_iterations", number(iter)},
	};
	read_params(in, p, true, n);
	if (!(*eps > 0)) bad("bisection.absolute_error", std::to_string(*eps));
	if (!(*iter > 0)) bad("bisection.max_iterations", std::to_string(*iter));
}

void read_nit(std::istream& in, ArConfig* c) {
	double acf_ab[2] = {0, 1}, acf_eps = 1e-6;
	int acf_iter = 100, nodes = 100, max_int = 12, max_exp = 10;
	std::map<std::string, Reader> p = {
	    {"distribution",
	     [c](std::istream& s, const std::string& k) {
		     const std::string d = read_word(s);
		     if (d == "gram_charlier") {
			     c->nit_dist = ARMA_NIT_GRAM_CHARLIER;
			     std::map<std::string, Reader> q = {{"skewness", number(&c->nit_params[0])},
			                                        {"kurtosis", number(&c->nit_params[1])}};
			     read_params(s, q, true, k);
		     } else if (d == "skew_normal") {
			     c->nit_dist = ARMA_NIT_SKEW_NORMAL;
			     std::map<std::string, Reader> q = {{"mean", number(&c->nit_params[0])},
			                                        {"stdev", number(&c->nit_params[1])},
			                                        {"alpha", number(&c->nit_params[2])}};
			     read_params(s, q, true, k);
		     } else {
			     throw Error{ARMA_EINVAL, "Invalid distribution: " + d};
		     }
	     }},
	    {"max_interpolation_order", number(&max_int)},
	    {"interpolation_nodes", number(&nodes)},
	    {"max_expansion_order", number(&max_exp)},
	    {"cdf_solver",
	     [c](std::istream& s, const std::string& k) {
		     read_bisection(s, c->cdf_interval, &c->cdf_eps, &c->cdf_iter, k);
	     }},
	    {"acf_solver",
	     [&](std::istream& s, const std::string& k) {
		     read_bisection(s, acf_ab, &acf_eps, &acf_iter, k);
	     }},
	};
	read_params(in, p, true, "nit_transform");
	if (nodes <= 0 || max_int <= 0 || max_exp <= 0) bad("nit_transform", "non-positive order");
}

void read_ar(std::istream& in, ArConfig* c) {
	std::map<std::string, Reader> p = {
	    {"out_grid", [c](std::istream& s, const std::string& k) { read_grid(s, &c->out_grid, k); }},
	    {"no_seed", number(&c->no_seed)},
	    {"transform",
	     [c](std::istream& s, const std::string&) {
		     const std::string name = read_word(s);
		     if (name == "nit") {
			     c->nit = true;
			     read_nit(s, c);
		     } else if (name == "none") {
			     c->nit = false;
		     } else {
			     throw Error{ARMA_EINVAL, "Invalid transform: " + name};
		     }
	     }},
	    {"acf",
	     [c](std::istream& s, const std::string& k) {
		     // Without `grid` this is the reference's ACF_generator (a plain
		     // wave group: func, amplitude, velocity, alpha, beta = wave
		     // numbers, nwaves, shape; src/generator/acf_generator.cc:250-263);
		     // with `grid` the analytic standing / propagating ACF of
		     // ACF_wrapper (src/bits/acf_wrapper.cc:41-70).
		     std::string func;
		     bool has_grid = false, has_wave_keys = false;
		     const double nan = std::numeric_limits<double>::quiet_NaN();
		     double amp = nan, vel = nan, al[3] = {nan, nan, nan}, be[2] = {nan, nan};
		     double nw[3] = {nan, nan, nan};
		     int shp[3] = {-1, -1, -1};
		     std::map<std::string, Reader> q = {
		         {"grid", [c, &has_grid](std::istream& t, const std::string& kk) {
			          read_grid(t, &c->acf_grid, kk);
			          has_grid = true;
		          }},
		         {"func", [&func](std::istream& t, const std::string&) { func = read_word(t); }},
		         {"amplitude", number(&amp)},
		         {"velocity", number(&vel)},
		         {"alpha", tuple<double, 3>(al)},
		         {"beta", tuple<double, 2>(be)},
		         {"nwaves", [&](std::istream& t, const std::string& kk) {
			          read_tuple<double, 3>(t, nw, kk);
			          has_wave_keys = true;
		          }},
		         {"shape", [&](std::istream& t, const std::string& kk) {
			          read_tuple<int, 3>(t, shp, kk);
			          has_wave_keys = true;
		          }},
		     };
		     read_params(s, q, true, k);
		     auto pick = [](double v, double dflt) { return std::isnan(v) ? dflt : v; };
		     if (has_grid) {
			     if (has_wave_keys)
				     throw Error{ARMA_EINVAL, "Bad \"acf\": grid with nwaves/shape"};
			     c->amplitude = pick(amp, 1.0);
			     c->velocity = pick(vel, 0.0);
			     for (int i = 0; i < 3; ++i) c->alpha[i] = pick(al[i], 0.0);
			     for (int i = 0; i < 2; ++i) c->beta[i] = pick(be[i], 0.0);
			     if (func == "standing_wave") c->acf_kind = ARMA_ACF_STANDING;
			     else if (func == "propagating_wave") c->acf_kind = ARMA_ACF_PROPAGATING;
			     else throw Error{ARMA_EINVAL, "Bad ACF function name: \"" + func + "\""};
		     } else {
			     EmpiricalAcf& w = c->wave;
			     if (func.empty() || func == "cos") w.func = 1;
			     else if (func == "sin") w.func = 0;
			     else if (func == "stokes") w.func = 2;
			     else if (func == "standing_wave") w.func = 3;
			     else throw Error{ARMA_EINVAL, "Invalid plain wave function: " + func};
			     w.amplitude = pick(amp, 1.0);
			     w.velocity = pick(vel, 1.0);
			     for (int i = 0; i < 3; ++i) w.alpha[i] = pick(al[i], 0.06);
			     w.wavenum[0] = pick(be[0], 0.8);
			     w.wavenum[1] = pick(be[1], 0.0);
			     for (int i = 0; i < 3; ++i) w.nwaves[i] = pick(nw[i], 1.5);
			     for (int i = 0; i < 3; ++i) w.shape[i] = shp[i] < 0 ? 16 : shp[i];
			     for (int i = 0; i < 3; ++i)
				     if (w.shape[i] > 64) bad(k, "shape above 64");
			     c->acf_empirical = true;
			     c->acf_kind = -2;
		     }
	     }},
	    {"output", [c](std::istream& s, const std::string& k) { c->output = read_flags(s, k); }},
	    {"order", tuple<int, 3>(c->order)},
	    {"validate", number(&c->validate)},
	    {"algorithm", [c](std::istream& s, const std::string&) { c->algorithm = read_word(s); }},
	    {"partition", tuple<int, 3>(c->partition)},
	    // extensions
	    {"seed",
	     [c](std::istream& s, const std::string& k) {
		     if (!(s >> c->seed)) bad(k, "expecting an unsigned integer");
		     c->has_seed = true;
	     }},
	    {"mt_file", [c](std::istream& s, const std::string&) { c->mt_file = read_word(s); }},
	    {"precision",
	     [c](std::istream& s, const std::string& k) {
		     const std::string w = read_word(s);
		     if (w == "fp64") c->precision = ARMA_FP64;
		     else if (w == "fp32c") c->precision = ARMA_FP32C;
		     else bad(k, w);
	     }},
	};
	read_params(in, p, true, c->ma ? "MA" : "AR");
	if (c->ma) {
		// MA_algorithm names (src/ma_algorithm.cc:7-21)
		if (c->algorithm != "fixed_point_iteration" && c->algorithm != "newton_raphson")
			throw Error{ARMA_EINVAL, "Invalid MA algorithm: " + c->algorithm};
	} else if (c->algorithm != "gauss_elimination" && c->algorithm != "choi_recursive") {
		throw Error{ARMA_EINVAL, "bad AR algorithm"};
	}
	if (c->acf_kind == -1) throw Error{ARMA_EINVAL, "Bad \"acf\": missing"};
	for (int i = 0; i < 3; ++i)
		if (c->out_grid.n[i] <= 0) bad("out_grid", "missing");
}

struct SolverConfig {
	Domain2 domain;
	double depth = 0;
	std::vector<double> z_levels;  // extension: explicit depth levels
};

void read_linear(std::istream& in, SolverConfig* c) {
	Domain2 wnmax;
	std::map<std::string, Reader> p = {
	    {"wnmax", [&wnmax](std::istream& s, const std::string& k) { read_domain(s, &wnmax, k); }},
	    {"depth", real_or_inf(&c->depth)},
	    {"domain", [c](std::istream& s, const std::string& k) { read_domain(s, &c->domain, k); }},
	    {"z_levels",
	     [c](std::istream& s, const std::string& k) {
		     if (!expect(s, '[')) bad(k, "expecting \"[\"");
		     c->z_levels.clear();
		     double v;
		     while (s >> v) {
			     c->z_levels.push_back(v);
			     if (expect(s, ']')) return;
			     if (!expect(s, ',')) bad(k, "expecting \",\"");
		     }
		     bad(k, "expecting \"]\"");
	     }},
	};
	read_params(in, p, true, "velocity_potential_solver");
	if (!(c->depth > 0)) bad("depth", "must be positive (or inf)");
	if (c->domain.lo[1] < -c->depth) throw Error{ARMA_EINVAL, "min(z) is less than -h"};
}

// ------------------------------------------------------------- the driver
struct Driver {
	std::string model_name, solver_name;
	ArConfig ar;
	SolverConfig solver;
	bool has_solver = false;
	// results
	std::vector<double> acf;
	int acf_shape[3] = {0, 0, 0};
	double acf_delta[3] = {1, 1, 1};
	std::vector<double> phi;
	double var_wn = 0;
	int shape[3] = {0, 0, 0};
	double delta[3] = {1, 1, 1};
	std::vector<double> zeta;
	std::vector<double> vel;  // (ntd, nz, nx, ny)
	std::vector<double> vel_t, vel_z;
	// where files written while generating go (the reference: the working
	// directory); zeta.bin of an AR model is written then, not by write_all
	std::string out_dir;
	bool bin_written = false;
};

namespace {

// The registry: every name the reference registers; the ones this library
// does not build report ARMA_ENOTSUP (src/register_all.hh:47-68).
const std::map<std::string, bool>& model_registry() {
	static const std::map<std::string, bool> m = {
	    {"AR", true}, {"MA", true}, {"ARMA", false}, {"plain_wave", false}, {"LH", false}};
	return m;
}
const std::map<std::string, bool>& solver_registry() {
	static const std::map<std::string, bool> m = {
	    {"linear", true}, {"plain", false}, {"high_amplitude", true}, {"small_amplitude", false}};
	return m;
}

void parse_driver(std::istream& in, Driver* d) {
	std::map<std::string, Reader> p = {
	    {"model",
	     [d](std::istream& s, const std::string&) {
		     d->model_name = read_word(s);
		     auto it = model_registry().find(d->model_name);
		     if (it == model_registry().end()) throw Error{ARMA_EINVAL, "bad object"};
		     if (!it->second)
			     throw Error{ARMA_ENOTSUP, "model \"" + d->model_name + "\" is not built"};
		     if (d->model_name == "MA") {
			     d->ar.ma = true;
			     d->ar.algorithm = "fixed_point_iteration";
		     }
		     read_ar(s, &d->ar);
	     }},
	    {"velocity_potential_solver",
	     [d](std::istream& s, const std::string&) {
		     d->solver_name = read_word(s);
		     auto it = solver_registry().find(d->solver_name);
		     if (it == solver_registry().end()) throw Error{ARMA_EINVAL, "bad object"};
		     if (!it->second)
			     throw Error{ARMA_ENOTSUP, "solver \"" + d->solver_name + "\" is not built"};
		     read_linear(s, &d->solver);
		     d->has_solver = true;
	     }},
	};
	read_params(in, p, false, "driver");
	if (!d->has_solver) throw Error{ARMA_EINVAL, "Bad \"velocity_potential_solver\": null"};
	if (d->model_name.empty()) throw Error{ARMA_EINVAL, "Bad \"generator\": null"};
}

// Shapes fixed by the configuration alone (src/generator/basic_arma_model.cc:
// 56-66, src/generator/ar_model.cc:102-105).
void finalise(Driver* d) {
	ArConfig& a = d->ar;
	if (a.acf_empirical) {  // the wave-group ACF is fixed by the configuration
		d->acf = empirical_acf(a.wave, d->acf_shape, d->acf_delta);
	} else {
		for (int i = 0; i < 3; ++i) {
			d->acf_shape[i] = a.acf_grid.n[i];
			d->acf_delta[i] = a.acf_grid.delta(i);
			if (a.acf_grid.n[i] <= 0) bad("acf.grid", "missing");
		}
	}
	// all(order) == 0 in the reference: any zero component takes the ACF shape
	if (a.order[0] == 0 || a.order[1] == 0 || a.order[2] == 0)
		for (int i = 0; i < 3; ++i) a.order[i] = d->acf_shape[i];
	for (int i = 0; i < 3; ++i)
		if (a.order[i] <= 0 || a.order[i] > d->acf_shape[i])
			throw Error{ARMA_EINVAL, a.ma ? "bad order" : "bad AR model order"};
	// output grid lengths := acf.delta * npatches * 2 pi, i.e. the output
	// step is 2 pi times the ACF step
	for (int i = 0; i < 3; ++i) {
		d->shape[i] = a.out_grid.n[i];
		d->delta[i] = d->acf_delta[i] * kTwoPi;
	}
}

}  // namespace

namespace {
// The reference's writer thread (src/generator/ar_model_parallel.cc:112-145):
// with the `binary` flag, an AR model's surface goes to zeta.bin in t-slabs,
// network byte order, as the generation completes them.  The reference joins
// the writer before it renormalises the surface and applies the NIT
// (src/generator/ar_model_parallel.cc:196-198, src/generator/basic_arma_model.cc:
// 100-110), so the file holds the surface as generated, and write_all does not
// write it again (src/arma_driver.cc:41-46, src/generator/ar_model.hh:59-62).
// Here the device->host copies of the slabs run on the context's copy stream
// into page-locked memory and a host thread converts and writes each slab as
// its copy completes, while the device goes on with the renormalisation.
class SlabWriter {
public:
	SlabWriter(Ctx* c, const void* d_src, const int shape[3], size_t es, const std::string& path)
	    : es_(es), path_(path) {
		const size_t slice = size_t(shape[1]) * shape[2];
		n_ = size_t(shape[0]) * slice;
		const size_t per = std::max<size_t>(1, (size_t(4) << 20) / std::max<size_t>(slice, 1));
		if (!c->copy_stream)
			ARMA_CUDA_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
		ARMA_CUDA_TRY(cudaHostAlloc(&stage_, std::max<size_t>(n_ * es_, 1), cudaHostAllocDefault));
		cudaEvent_t ready;
		ARMA_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
		events_.push_back(ready);
		ARMA_CUDA_TRY(cudaEventRecord(ready, c->stream));
		ARMA_CUDA_TRY(cudaStreamWaitEvent(c->copy_stream, ready, 0));
		for (size_t t0 = 0; t0 < size_t(shape[0]); t0 += per) {
			const size_t off = t0 * slice, cnt = std::min(per, size_t(shape[0]) - t0) * slice;
			ARMA_CUDA_TRY(copy_async(c, static_cast<char*>(stage_) + off * es_,
			                         static_cast<const char*>(d_src) + off * es_, cnt * es_,
			                         cudaMemcpyDeviceToHost, c->copy_stream));
			cudaEvent_t e;
			ARMA_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
			events_.push_back(e);
			ARMA_CUDA_TRY(cudaEventRecord(e, c->copy_stream));
			slabs_.push_back({off, cnt});
		}
		thread_ = std::thread([this] { run(); });
	}
	~SlabWriter() {
		if (thread_.joinable()) thread_.join();
		for (cudaEvent_t e : events_) cudaEventDestroy(e);
		if (stage_) cudaFreeHost(stage_);
	}
	// waits for the writer; throws what it met
	void finish() {
		if (thread_.joinable()) thread_.join();
		if (!error_.empty()) throw Error{error_code_, error_};
	}

private:
	void run() {
		std::ofstream out(path_, std::ios::binary);
		if (!out) {
			error_code_ = ARMA_EIO;
			error_ = "cannot write " + path_;
		}
		std::vector<unsigned char> buf;
		for (size_t k = 0; k < slabs_.size(); ++k) {
			if (cudaEventSynchronize(events_[k + 1]) != cudaSuccess) {
				error_code_ = ARMA_ECUDA;
				error_ = "zeta.bin: device->host copy failed";
				return;
			}
			if (!error_.empty()) continue;  // drain the copies, write nothing
			const size_t off = slabs_[k].first, cnt = slabs_[k].second;
			buf.resize(cnt * 8);
			for (size_t i = 0; i < cnt; ++i) {
				double v;
				if (es_ == 8) std::memcpy(&v, static_cast<char*>(stage_) + (off + i) * 8, 8);
				else {
					float f;
					std::memcpy(&f, static_cast<char*>(stage_) + (off + i) * 4, 4);
					v = f;
				}
				unsigned char b[8];
				std::memcpy(b, &v, 8);
				for (int q = 0; q < 8; ++q) buf[i * 8 + q] = b[7 - q];  // network byte order
			}
			out.write(reinterpret_cast<const char*>(buf.data()), std::streamsize(buf.size()));
			if (!out) {
				error_code_ = ARMA_EIO;
				error_ = "cannot write " + path_;
			}
		}
	}

	size_t es_, n_ = 0;
	std::string path_;
	void* stage_ = nullptr;
	std::vector<cudaEvent_t> events_;
	std::vector<std::pair<size_t, size_t>> slabs_;
	std::thread thread_;
	int error_code_ = ARMA_OK;
	std::string error_;
};
}  // namespace

void driver_set_output_dir(Driver* d, const std::string& dir) { d->out_dir = dir; }

// generate: ACF -> order -> grid rescale -> fit (AR: Yule-Walker, MA: fixed
// point) -> noise -> AR or MA filter -> renorm -> NIT
void driver_generate(Ctx* c, Driver* d) {
	ArConfig& a = d->ar;
	double adelta[3] = {d->acf_delta[0], d->acf_delta[1], d->acf_delta[2]};
	if (!a.acf_empirical) {
		d->acf.resize(size_t(d->acf_shape[0]) * d->acf_shape[1] * d->acf_shape[2]);
		acf_eval(a.acf_kind, a.amplitude, a.velocity, a.alpha, a.beta, adelta, d->acf_shape,
		         d->acf.data());
	}
	// The reference NIT-transforms a copy of the ACF and discards it
	// (src/generator/basic_arma_model.cc:74-79): the fit uses the Gaussian ACF.
	if (a.ma) {
		// MA_model::determine_coefficients / fixed_point_iteration
		// (src/generator/ma_model.cc:96-107, 153-163)
		if (a.algorithm != "fixed_point_iteration")
			throw Error{ARMA_ENOTSUP, "only fixed_point_iteration is supported"};
		const int rc = ma_fit_fixed_point(d->acf.data(), d->acf_shape, a.order, MaFitOptions{},
		                                  &d->phi, &d->var_wn, nullptr, nullptr);
		if (rc == 1) throw Error{ARMA_EINVAL, "bad order"};
		if (rc == 2) throw Error{ARMA_ENUMERIC, "bad MA model coefficients"};
		if (rc == 3) throw Error{ARMA_ENUMERIC, "bad white noise variance"};
		d->var_wn = ma_white_noise_variance(d->acf.data(), d->phi.data(), a.order);
	} else if (a.algorithm == "choi_recursive") {
		// determine_coefficients_choi (src/generator/ar_model.cc:136-152): the
		// order-recursive solver on the ACF table, maximum order max(order),
		// variance tolerance 1e-6, chopped; the model's order replaces the
		// configured one and var_wn is recomputed from phi
		const int n = d->acf_shape[0];
		if (d->acf_shape[1] != n || d->acf_shape[2] != n)
			throw Error{ARMA_EINVAL, "ACF is not square"};
		const int mo = std::max(a.order[0], std::max(a.order[1], a.order[2]));
		double solver_var = 0.0;
		const int rc = fit_choi(d->acf.data(), n, mo, true, 1e-6, true, 1e-10, &d->phi, a.order,
		                        &solver_var);
		if (rc == 2) throw Error{ARMA_ENUMERIC, "singular Yule-Walker block"};
		if (rc != 0) throw Error{ARMA_EINVAL, "bad AR model order"};
		d->var_wn = ar_white_noise_variance(d->acf.data(), d->acf_shape, d->phi.data(), a.order);
	} else {
		const int P0 = a.order[0] * a.order[1] * a.order[2];
		d->phi.assign(P0, 0.0);
		const int info =
		    a.acf_empirical
		        ? fit_gauss_table(d->acf.data(), d->acf_shape, a.order, ARMA_FIT_CHOLESKY,
		                          d->phi.data(), &d->var_wn)
		        : fit_analytic(a.acf_kind, a.amplitude, a.velocity, a.alpha, a.beta, adelta, a.order,
		                       d->phi.data(), &d->var_wn);
		if (info != 0)
			throw Error{ARMA_ENUMERIC, "Yule-Walker matrix is not positive definite"};
	}
	const int P = a.order[0] * a.order[1] * a.order[2];
	// validate_process on the fitted coefficients (src/generator/basic_arma_model.cc:
	// 92-96, src/generator/ar_model.cc:64-68), before the noise
	if (a.validate) {
		int bad = 0;
		const int rc = validate_ar_process(d->phi.data(), P, &bad);
		if (rc == 1) throw Error{ARMA_ENUMERIC, "leading term of polynomial must be non-zero"};
		if (rc == 2) throw Error{ARMA_ENUMERIC, "root solving qr method failed to converge"};
		if (rc == 3)
			throw Error{ARMA_EINVAL,
			            "AR/MA process is not stationary/invertible: some roots lie inside unit "
			            "circle or on its borderline."};
	}
	if (d->var_wn < 0.0) throw Error{ARMA_EINVAL, "variance is less than zero"};
	arma_mt_params mt;
	{
		std::ifstream f(a.mt_file, std::ios::binary);
		if (!f)
			throw Error{ARMA_EIO, "Mersenne Twister configuration file not found: " + a.mt_file};
	}
	if (arma_mt_file_read(a.mt_file.c_str(), 0, &mt) != ARMA_OK)
		throw Error{ARMA_EPRNG, "bad number of MT configs"};
	uint32_t seed = 0;
	if (!a.no_seed)
		seed = a.has_seed ? a.seed
		                  : uint32_t(std::chrono::high_resolution_clock::now().time_since_epoch().count());
	const size_t n = size_t(d->shape[0]) * d->shape[1] * d->shape[2];
	const size_t es = a.precision == ARMA_FP64 ? 8 : 4;
	void* dz = scratch_take(c, n * es);
	arma_surface s{};
	for (int i = 0; i < 3; ++i) {
		s.shape[i] = d->shape[i];
		s.order[i] = a.order[i];
	}
	s.phi = d->phi.data();
	s.var_wn = d->var_wn;
	s.acf0 = d->acf[0];
	s.mt = mt;
	s.seed = seed;
	s.d_zeta = dz;
	d->bin_written = false;
	const bool stream_bin = !a.ma && (a.output & (1u << F_BINARY));
	if (a.ma) {
		ma_generate_device(c, &s, 1, a.precision);
	} else if (!stream_bin) {
		batch_generate_device(c, &s, 1, a.precision);
	} else {
		// the surface as generated, then its renormalisation on a copy while
		// the writer streams the generated one to zeta.bin
		s.acf0 = 0.0;
		batch_generate_device(c, &s, 1, a.precision);
		SlabWriter w(c, dz, d->shape, es, (d->out_dir.empty() ? "" : d->out_dir + "/") + "zeta.bin");
		void* dz2 = scratch_take(c, n * es);
		ARMA_CUDA_TRY(cudaMemcpyAsync(dz2, dz, n * es, cudaMemcpyDeviceToDevice, c->stream));
		dz = dz2;
		auto* d_scale = static_cast<double*>(scratch_take(c, sizeof(double)));
		RenormSpec r{dz, {d->shape[0], d->shape[1], d->shape[2]}, d->acf[0], d_scale};
		launch_renorm_batch(c, {r}, a.precision);
		w.finish();
		d->bin_written = true;
	}
	if (a.nit) {
		launch_nit_bisection(c, a.nit_dist, a.nit_params, std::sqrt(d->acf[0]), a.cdf_interval[0],
		                     a.cdf_interval[1], a.cdf_eps, a.cdf_iter, n, a.precision, dz);
	}
	d->zeta.resize(n);
	if (a.precision == ARMA_FP64) {
		ARMA_CUDA_TRY(cudaMemcpyAsync(d->zeta.data(), dz, n * 8, cudaMemcpyDeviceToHost, c->stream));
		ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
	} else {
		std::vector<float> tmp(n);
		ARMA_CUDA_TRY(cudaMemcpyAsync(tmp.data(), dz, n * 4, cudaMemcpyDeviceToHost, c->stream));
		ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
		for (size_t i = 0; i < n; ++i) d->zeta[i] = tmp[i];
	}
}

// velocity: domain t coordinates truncated to slice indices, z from the
// domain (or z_levels), (ntd, nz, nx, ny) FP64 result
void driver_velocity(Ctx* c, Driver* d) {
	if (!d->has_solver) throw Error{ARMA_EINVAL, "Bad \"velocity_potential_solver\": null"};
	const Domain2& dm = d->solver.domain;
	std::vector<int> tidx;
	d->vel_t.clear();
	d->vel_z.clear();
	for (int i = 0; i < dm.n[0]; ++i) {
		const double t = dm.at(i, 0);
		d->vel_t.push_back(t);
		tidx.push_back(int(t));
	}
	if (!d->solver.z_levels.empty()) {
		d->vel_z = d->solver.z_levels;
	} else {
		for (int j = 0; j < dm.n[1]; ++j) d->vel_z.push_back(dm.at(j, 1));
	}
	const size_t n = d->zeta.size();
	const size_t n2 = size_t(d->shape[1]) * d->shape[2];
	double* dz = static_cast<double*>(scratch_take(c, n * 8));
	double* dout = static_cast<double*>(scratch_take(c, n2 * tidx.size() * d->vel_z.size() * 8));
	ARMA_CUDA_TRY(cudaMemcpyAsync(dz, d->zeta.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
	launch_velocity_linear(c, dz, d->shape, ARMA_FP64, d->delta, d->solver.depth, d->vel_z.data(),
	                       int(d->vel_z.size()), tidx.data(), int(tidx.size()), dout,
	                       d->solver_name == "high_amplitude" ? 1 : 0);
	d->vel.resize(n2 * tidx.size() * d->vel_z.size());
	ARMA_CUDA_TRY(cudaMemcpyAsync(d->vel.data(), dout, d->vel.size() * 8, cudaMemcpyDeviceToHost,
	                              c->stream));
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
}

namespace {

// blitz text layout of an N-d array: the index ranges, then the values, one
// innermost row per line.
void write_blitz(const std::string& path, const double* v, const std::vector<int>& ext) {
	std::ofstream out(path);
	if (!out) throw Error{ARMA_EIO, "cannot write " + path};
	for (size_t i = 0; i < ext.size(); ++i) {
		out << '(' << 0 << ',' << ext[i] - 1 << ')';
		if (i + 1 != ext.size()) out << " x ";
	}
	out << "\n[ ";
	size_t n = 1;
	for (int e : ext) n *= size_t(e);
	const size_t row = size_t(ext.back());
	for (size_t i = 0; i < n; ++i) {
		out << v[i] << ' ';
		if ((i + 1) % row == 0 && i + 1 != n) out << "\n  ";
	}
	out << "]\n";
}

}  // namespace

// Reference: ARMA_driver::write_all (src/arma_driver.cc:121-130) with
// write_wavy_surface / write_velocity_potentials (:29-69): only when the
// "surface" flag is set; zeta / zeta.csv / zeta.bin, phi / phi.csv.
void driver_write(Driver* d, const std::string& dir) {
	const unsigned f = d->ar.output;
	if (!(f & (1u << F_SURFACE))) return;
	const std::string pre = dir.empty() ? "" : dir + "/";
	const int nt = d->shape[0], nx = d->shape[1], ny = d->shape[2];
	if (f & (1u << F_BLITZ)) write_blitz(pre + "zeta", d->zeta.data(), {nt, nx, ny});
	if (f & (1u << F_CSV)) {
		std::ofstream out(pre + "zeta.csv");
		if (!out) throw Error{ARMA_EIO, "cannot write " + pre + "zeta.csv"};
		out << "t,x,y,z\n";
		for (int i = 0; i < nt; ++i)
			for (int j = 0; j < nx; ++j)
				for (int k = 0; k < ny; ++k)
					out << i << ',' << d->delta[1] * j << ',' << d->delta[2] * k << ','
					    << d->zeta[(size_t(i) * nx + j) * ny + k] << '\n';
	}
	if ((f & (1u << F_BINARY)) && !d->bin_written) {
		std::ofstream out(pre + "zeta.bin", std::ios::binary);
		if (!out) throw Error{ARMA_EIO, "cannot write " + pre + "zeta.bin"};
		for (double v : d->zeta) {  // network byte order
			unsigned char b[8];
			std::memcpy(b, &v, 8);
			for (int k = 0; k < 4; ++k) std::swap(b[k], b[7 - k]);
			out.write(reinterpret_cast<const char*>(b), 8);
		}
	}
	if (!d->vel.empty()) {
		const int ntd = int(d->vel_t.size()), nz = int(d->vel_z.size());
		if (f & (1u << F_BLITZ)) write_blitz(pre + "phi", d->vel.data(), {ntd, nz, nx, ny});
		if (f & (1u << F_CSV)) {
			std::ofstream out(pre + "phi.csv");
			if (!out) throw Error{ARMA_EIO, "cannot write " + pre + "phi.csv"};
			out << "t,z,x,y,phi\n";
			for (int i = 0; i < ntd; ++i)
				for (int j = 0; j < nz; ++j)
					for (int k = 0; k < nx; ++k)
						for (int l = 0; l < ny; ++l)
							out << d->vel_t[i] << ',' << d->vel_z[j] << ',' << d->delta[1] * k << ','
							    << d->delta[2] * l << ','
							    << d->vel[((size_t(i) * nz + j) * nx + k) * ny + l] << '\n';
		}
	}
}

void driver_info(const Driver* d, int shape[3], double delta[3], int order[3], double* var_wn,
                 int vshape[4], unsigned* oflags) {
	if (oflags) *oflags = d->ar.output;
	for (int i = 0; i < 3; ++i) {
		if (shape) shape[i] = d->shape[i];
		if (delta) delta[i] = d->delta[i];
		if (order) order[i] = d->ar.order[i];
	}
	if (var_wn) *var_wn = d->var_wn;
	if (vshape) {
		vshape[0] = int(d->vel_t.size());
		vshape[1] = int(d->vel_z.size());
		vshape[2] = d->vel.empty() ? 0 : d->shape[1];
		vshape[3] = d->vel.empty() ? 0 : d->shape[2];
	}
}

void driver_acf(const Driver* d, int shape[3], double delta[3], const double** data) {
	for (int i = 0; i < 3; ++i) {
		shape[i] = d->acf_shape[i];
		delta[i] = d->acf_delta[i];
	}
	*data = d->acf.empty() ? nullptr : d->acf.data();
}

const double* driver_zeta(const Driver* d) { return d->zeta.empty() ? nullptr : d->zeta.data(); }
const double* driver_phi(const Driver* d) { return d->phi.empty() ? nullptr : d->phi.data(); }
const double* driver_velocity_data(const Driver* d) {
	return d->vel.empty() ? nullptr : d->vel.data();
}

Driver* driver_open(const std::string& text) {
	std::unique_ptr<Driver> d(new Driver());
	std::istringstream in(text);
	parse_driver(in, d.get());
	finalise(d.get());
	return d.release();
}

void driver_close(Driver* d) { delete d; }

}  // namespace armab
