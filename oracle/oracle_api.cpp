// oracle_api.cpp -- C entry points of the CPU oracle (test infrastructure only;
// see oracle.hpp).  Arrays crossing this boundary use the reference layout
// a(nv,i,j,k): variable fastest, then i, j, k.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "oracle.hpp"

using orc::State;

int orc::g_pow_mode = 0;

extern "C" {

// Selects the power function of the step (0: the C library's pow, 1: rg_pow,
// see orc::fpow); returns the previous mode.  Process-wide.
int orc_set_pow_mode(int mode) {
  const int old = orc::g_pow_mode;
  orc::g_pow_mode = mode ? 1 : 0;
  return old;
}

// x[i]**y[i] by either power function, for the accuracy tests of rg_pow.
void orc_pow_eval(const double* x, const double* y, double* out, long long n, int mode) {
  for (long long i = 0; i < n; ++i) out[i] = mode ? rgm::pow(x[i], y[i]) : std::pow(x[i], y[i]);
}

void* orc_create(const orc_params* p) {
  State* s = new State();
  s->p = *p;
  s->imax = p->imax; s->jmax = p->jmax; s->kmax = p->kmax;
  s->ncell = (size_t)p->imax * p->jmax * p->kmax;
  // ghost widths (main.f90:176-199): second-order schemes nm0 = 2, five-point schemes nm0 = 3,
  // PPM nm0 = 4; constrained transport nm1 = nm0 + ict
  const int r = p->irec;
  s->nm0 = (r == 1 || r == 2 || r == 3 || r == 11 || r == 12 || r == 13) ? 2 : (r == 5 ? 4 : 3);
  s->nm1 = s->nm0 + p->ict;
  orc::grid(*s);
  orc::coord1(*s);
  orc::calchrist(*s);
  const size_t n9 = s->ncell * orc::NV;
  for (auto* v : {&s->uu, &s->uo, &s->uh, &s->us, &s->un, &s->uri, &s->urio, &s->uriir, &s->uriil,
                  &s->urijr, &s->urijl, &s->urikr, &s->urikl, &s->uuir, &s->uuil, &s->uujr, &s->uujl,
                  &s->uukr, &s->uukl, &s->wwir, &s->wwil, &s->wwjr, &s->wwjl, &s->wwkr, &s->wwkl})
    v->assign(n9, 0.0);
  s->ww.assign(3 * n9, 0.0);
  s->sf.assign(4 * s->ncell, 0.0);
  for (auto* v : {&s->cmaxi, &s->cmini, &s->cmaxj, &s->cminj, &s->cmaxk, &s->cmink}) v->assign(s->ncell, 0.0);
  return s;
}

void orc_destroy(void* h) { delete static_cast<State*>(h); }

int orc_nm1(void* h) { return static_cast<State*>(h)->nm1; }

// mdtorus1 followed by the copies of main.f90:530-548
void orc_ic_torus(void* h, unsigned long long seed, double amp, double rin, double rmax, double beta,
                  double kappa) {
  State* s = static_cast<State*>(h);
  orc::mdtorus1(*s, seed, amp, rin, rmax, beta, kappa);
}

// seeded Riemann tube (pattern of mdshoctub, mdgrmhd.f90:56-118)
void orc_ic_tube(void* h, unsigned long long seed, unsigned long long tube) {
  orc::mdtube(*static_cast<State*>(h), seed, tube);
}

void orc_set_prims(void* h, const double* uri) {
  State* s = static_cast<State*>(h);
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
}

void orc_get_prims(void* h, double* uri) {
  State* s = static_cast<State*>(h);
  std::memcpy(uri, s->uri.data(), s->uri.size() * sizeof(double));
}

void orc_get_cons(void* h, double* uu) {
  State* s = static_cast<State*>(h);
  std::memcpy(uu, s->uu.data(), s->uu.size() * sizeof(double));
}

// main.f90:530-548: conserved from primitives, time = 0
void orc_init_cons(void* h) {
  State* s = static_cast<State*>(h);
  orc::caluu1(*s, s->uri, s->uu);
  s->uo = s->uu;
  s->urio = s->uri;
  s->time = 0.0; s->timeh = 0.0; s->it = 0;
}

// Runs up to nsteps passes of the time loop; stops early (returns the count
// done) when the loop-top time exceeds tmax (main.f90:617-632).
int orc_step(void* h, int nsteps) {
  State* s = static_cast<State*>(h);
  for (int n = 0; n < nsteps; ++n) {
    if (s->timeh > s->p.tmax) return n;
    orc::step(*s);
  }
  return nsteps;
}

double orc_time(void* h) { return static_cast<State*>(h)->timeh; }
double orc_dt(void* h) { return static_cast<State*>(h)->dt; }
void orc_get_stats(void* h, orc_stats* out) { *out = static_cast<State*>(h)->st; }

// Per-routine hooks used by the parity tests ------------------------------

// caluu1 on the given primitives
void orc_caluu1(void* h, const double* uri, double* uu) {
  State* s = static_cast<State*>(h);
  std::vector<double> p(uri, uri + s->uri.size()), u(s->uu.size());
  orc::caluu1(*s, p, u);
  std::memcpy(uu, u.data(), u.size() * sizeof(double));
}

// rec2 + calcha + hll + ct on the given primitives; ww(3,nv,i,j,k) out
void orc_fluxes(void* h, const double* uri, double* ww) {
  State* s = static_cast<State*>(h);
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
  orc::rec2(*s);
  orc::calcha(*s);
  orc::hlle(*s);
  orc::ct(*s);
  std::memcpy(ww, s->ww.data(), s->ww.size() * sizeof(double));
}

// ct alone (ct.f90:4-27, the run's ict) on given primitives and fluxes ww(3,nv,i,j,k), in place
void orc_ct(void* h, const double* uri, double* ww) {
  State* s = static_cast<State*>(h);
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
  std::memcpy(s->ww.data(), ww, s->ww.size() * sizeof(double));
  orc::ct(*s);
  std::memcpy(ww, s->ww.data(), s->ww.size() * sizeof(double));
}

// rec2 alone on the given primitives: the six face-state arrays uriil,
// uriir, urijl, urijr, urikl, urikr (each 9 per cell, reference layout) out
void orc_rec2(void* h, const double* uri, double* faces) {
  State* s = static_cast<State*>(h);
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
  std::vector<double>* f[6] = {&s->uriil, &s->uriir, &s->urijl, &s->urijr, &s->urikl, &s->urikr};
  for (auto* v : f) std::fill(v->begin(), v->end(), 0.0);
  orc::rec2(*s);
  for (int m = 0; m < 6; ++m) std::memcpy(faces + m * s->uri.size(), f[m]->data(), s->uri.size() * sizeof(double));
}

// rec2 with its face conserved variables and fluxes (rec.f90:2-142: the
// reconstruction, then caluu3 and calflx3 per direction): six arrays each of
// face primitives, face conserved variables and face fluxes, in the order
// ?il, ?ir for ? = i, j, k (each 9 per cell, reference layout; entries the
// reference does not set are 0).  cons or flux may be null.
void orc_rec2_full(void* h, const double* uri, double* prims, double* cons, double* flux) {
  State* s = static_cast<State*>(h);
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
  std::vector<double>* f[3][6] = {{&s->uriil, &s->uriir, &s->urijl, &s->urijr, &s->urikl, &s->urikr},
                                  {&s->uuil, &s->uuir, &s->uujl, &s->uujr, &s->uukl, &s->uukr},
                                  {&s->wwil, &s->wwir, &s->wwjl, &s->wwjr, &s->wwkl, &s->wwkr}};
  for (auto& row : f)
    for (auto* v : row) std::fill(v->begin(), v->end(), 0.0);
  orc::rec2(*s);
  double* out[3] = {prims, cons, flux};
  const size_t n = s->uri.size();
  for (int a = 0; a < 3; ++a)
    if (out[a])
      for (int m = 0; m < 6; ++m) std::memcpy(out[a] + m * n, f[a][m]->data(), n * sizeof(double));
}

// calcha (calcha.f90:2-126) from given face primitives (six arrays as
// orc_rec2_full): cmaxi, cmini, cmaxj, cminj, cmaxk, cmink (one per cell each)
void orc_calcha(void* h, const double* prims, double* cha) {
  State* s = static_cast<State*>(h);
  std::vector<double>* f[6] = {&s->uriil, &s->uriir, &s->urijl, &s->urijr, &s->urikl, &s->urikr};
  const size_t n = s->uri.size();
  for (int m = 0; m < 6; ++m) std::memcpy(f[m]->data(), prims + m * n, n * sizeof(double));
  std::vector<double>* c[6] = {&s->cmaxi, &s->cmini, &s->cmaxj, &s->cminj, &s->cmaxk, &s->cmink};
  for (auto* v : c) std::fill(v->begin(), v->end(), 0.0);
  orc::calcha(*s);
  for (int m = 0; m < 6; ++m) std::memcpy(cha + m * s->ncell, c[m]->data(), s->ncell * sizeof(double));
}

// hll (hll.f90:47-192) from given face conserved variables, face fluxes and
// characteristic speeds: ww(3,nv,i,j,k) in/out (entries outside the hll
// range keep their values)
void orc_hll(void* h, const double* cons, const double* flux, const double* cha, double* ww) {
  State* s = static_cast<State*>(h);
  const size_t n = s->uri.size();
  std::vector<double>* u[6] = {&s->uuil, &s->uuir, &s->uujl, &s->uujr, &s->uukl, &s->uukr};
  std::vector<double>* w[6] = {&s->wwil, &s->wwir, &s->wwjl, &s->wwjr, &s->wwkl, &s->wwkr};
  std::vector<double>* c[6] = {&s->cmaxi, &s->cmini, &s->cmaxj, &s->cminj, &s->cmaxk, &s->cmink};
  for (int m = 0; m < 6; ++m) {
    std::memcpy(u[m]->data(), cons + m * n, n * sizeof(double));
    std::memcpy(w[m]->data(), flux + m * n, n * sizeof(double));
    std::memcpy(c[m]->data(), cha + m * s->ncell, s->ncell * sizeof(double));
  }
  std::memcpy(s->ww.data(), ww, s->ww.size() * sizeof(double));
  orc::hlle(*s);
  std::memcpy(ww, s->ww.data(), s->ww.size() * sizeof(double));
}

// recov1a over the interior: uu (in/out, uu(6) rewritten), uri (in: guess, out)
void orc_recov(void* h, double* uu, double* uri) {
  State* s = static_cast<State*>(h);
  std::vector<double> u(uu, uu + s->uu.size());
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
  orc::recov(*s, u);
  std::memcpy(uu, u.data(), u.size() * sizeof(double));
  std::memcpy(uri, s->uri.data(), s->uri.size() * sizeof(double));
}

// caltenr + calsf on every cell of the given primitives; sf(2:5,i,j,k) out
void orc_calsf(void* h, const double* uri, double* sf) {
  State* s = static_cast<State*>(h);
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
  orc::calsf_all(*s, true);
  std::memcpy(sf, s->sf.data(), s->sf.size() * sizeof(double));
}

// One RK3 stage (rkstage) with the given dt, ww, sf and conserved inputs:
// stage 1 uh from uu = ucur; stage 2 us from uo and uh = ucur; stage 3 un from
// uo and us = ucur.  unew is in/out (cells outside the interior keep theirs).
void orc_rkt(void* h, int stage, double dt, const double* ww, const double* uo, const double* ucur,
             const double* sf, double* unew) {
  State* s = static_cast<State*>(h);
  const size_t n = s->uu.size();
  s->dt = dt;
  std::memcpy(s->ww.data(), ww, s->ww.size() * sizeof(double));
  std::memcpy(s->sf.data(), sf, s->sf.size() * sizeof(double));
  std::vector<double>& in = (stage == 1) ? s->uu : (stage == 2 ? s->uh : s->us);
  std::vector<double>& out = (stage == 1) ? s->uh : (stage == 2 ? s->us : s->un);
  std::memcpy(in.data(), ucur, n * sizeof(double));
  if (stage > 1) std::memcpy(s->uo.data(), uo, n * sizeof(double));
  std::memcpy(out.data(), unew, n * sizeof(double));
  orc::rkstage(*s, stage);
  std::memcpy(unew, out.data(), n * sizeof(double));
}

// the output converter's derived quantities (7 per point) of the given
// primitives: every cell (jslice = 0) or the phi plane jslice
void orc_derived(void* h, const double* uri, int jslice, double* out) {
  State* s = static_cast<State*>(h);
  std::vector<double> u(uri, uri + s->uri.size());
  orc::derived(*s, u, jslice, out);
}

// cdtcfl4 on the given primitives
double orc_cdtcfl(void* h, const double* uri) {
  State* s = static_cast<State*>(h);
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
  return orc::cdtcfl4(*s);
}

// bnd4 + infchk + atmosphere1a + pminmax2b on uri (in/out) with urio
// One of bnd4 (which 0), infchk (1), atmosphere1a (2), pminmax2b (3) alone on
// uri in place, each with the reference's model condition (main.f90:860-878).
void orc_bnd_part(void* h, int which, double* uri, const double* urio) {
  State* s = static_cast<State*>(h);
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
  if (urio) std::memcpy(s->urio.data(), urio, s->urio.size() * sizeof(double));
  if (which == 0) orc::bnd4(*s);
  else if (which == 1) { if (s->p.model >= 7 && s->p.model <= 20) orc::infchk(*s); }
  else if (which == 2) { if (s->p.model >= 7 && s->p.model <= 15) orc::atmosphere1a(*s); }
  else orc::pminmax2b(*s);
  std::memcpy(uri, s->uri.data(), s->uri.size() * sizeof(double));
}

void orc_bnd_floor(void* h, double* uri, const double* urio) {
  State* s = static_cast<State*>(h);
  std::memcpy(s->uri.data(), uri, s->uri.size() * sizeof(double));
  std::memcpy(s->urio.data(), urio, s->urio.size() * sizeof(double));
  orc::bnd4(*s);
  if (s->p.model >= 7 && s->p.model <= 20) orc::infchk(*s);
  if (s->p.model >= 7 && s->p.model <= 15) orc::atmosphere1a(*s);
  orc::pminmax2b(*s);
  std::memcpy(uri, s->uri.data(), s->uri.size() * sizeof(double));
}

// Grid and metric arrays by name.  1D grid arrays: n = extent (1-based values
// copied to out[0..n-1]).  Metric per (i,k): 16 (gcov*/gcon*) or 1 (detg*)
// or 64 (christ) values per point, point index i-1 + imax*(k-1).
// output1 (restar.f90:91-185) for one rank holding the whole grid
// (is..ie = 1..imax etc.): gfortran sequential unformatted records, each
// framed by its 4-byte length: (time, myrank, npe), (is, ie, js, je, ks, ke),
// then for i, j, k (k fastest) x1(i), x2(j), x3(k), uri(1:9,i,j,k), detg.
// The coordinates are x?b for metric 403 and x? otherwise (main.f90:711-717);
// time is the loop-top time.  Returns 0 on success.
int orc_output1(void* h, const char* path, int myrank, int npe) {
  State* s = static_cast<State*>(h);
  FILE* f = std::fopen(path, "wb");
  if (!f) return 1;
  auto rec = [&](const void* d, uint32_t n) {
    return std::fwrite(&n, 4, 1, f) == 1 && std::fwrite(d, n, 1, f) == 1 && std::fwrite(&n, 4, 1, f) == 1;
  };
  unsigned char h1[16];
  std::memcpy(h1, &s->timeh, 8);
  std::memcpy(h1 + 8, &myrank, 4);
  std::memcpy(h1 + 12, &npe, 4);
  const int32_t h2[6] = {1, s->imax, 1, s->jmax, 1, s->kmax};
  bool ok = rec(h1, 16) && rec(h2, 24);
  const bool mks = (s->p.metric == 403);
  const std::vector<double>& X1 = mks ? s->x1b : s->x1;
  const std::vector<double>& X2 = mks ? s->x2b : s->x2;
  const std::vector<double>& X3 = mks ? s->x3b : s->x3;
  for (int i = 1; ok && i <= s->imax; ++i)
    for (int j = 1; ok && j <= s->jmax; ++j)
      for (int k = 1; ok && k <= s->kmax; ++k) {
        double v[13];
        v[0] = X1[i]; v[1] = X2[j]; v[2] = X3[k];
        for (int n = 1; n <= orc::NV; ++n) v[2 + n] = s->uri[s->a(n, i, j, k)];
        v[12] = s->detg[s->ik(i, k)];
        ok = rec(v, 104);
      }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? 0 : 1;
}

long long orc_get_array(void* h, const char* name, double* out, long long cap) {
  State* s = static_cast<State*>(h);
  const std::string n(name);
  auto vec1 = [&](const std::vector<double>& v, int len) -> long long {
    if (cap < len) return -1;
    for (int i = 1; i <= len; ++i) out[i - 1] = v[i];
    return len;
  };
  if (n == "x1") return vec1(s->x1, s->imax);
  if (n == "x1a") return vec1(s->x1a, s->imax);
  if (n == "x1b") return vec1(s->x1b, s->imax);
  if (n == "x1ab") return vec1(s->x1ab, s->imax);
  if (n == "x2a") return vec1(s->x2a, s->jmax);
  if (n == "x2b") return vec1(s->x2b, s->jmax);
  if (n == "x2ab") return vec1(s->x2ab, s->jmax);
  if (n == "x3ab") return vec1(s->x3ab, s->kmax);
  if (n == "dx1b") return vec1(s->dx1b, s->imax);
  if (n == "x2") return vec1(s->x2, s->jmax);
  if (n == "dx2b") return vec1(s->dx2b, s->jmax);
  if (n == "x3") return vec1(s->x3, s->kmax);
  if (n == "x3a") return vec1(s->x3a, s->kmax);
  if (n == "x3b") return vec1(s->x3b, s->kmax);
  if (n == "dx3b") return vec1(s->dx3b, s->kmax);
  const size_t nik = (size_t)s->imax * s->kmax;
  auto m4 = [&](const std::vector<orc::M4>& v) -> long long {
    if ((size_t)cap < 16 * nik) return -1;
    for (size_t q = 0; q < nik; ++q)
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) out[16 * q + 4 * a + b] = v[q].a[a][b];
    return (long long)(16 * nik);
  };
  auto sc = [&](const std::vector<double>& v) -> long long {
    if ((size_t)cap < nik) return -1;
    std::memcpy(out, v.data(), nik * sizeof(double));
    return (long long)nik;
  };
  if (n == "gcov") return m4(s->gcov);
  if (n == "gcon") return m4(s->gcon);
  if (n == "gcovi") return m4(s->gcovi);
  if (n == "gconi") return m4(s->gconi);
  if (n == "gcovk") return m4(s->gcovk);
  if (n == "gconk") return m4(s->gconk);
  if (n == "detg") return sc(s->detg);
  if (n == "detgi") return sc(s->detgi);
  if (n == "detgk") return sc(s->detgk);
  if (n == "christ") {
    if ((size_t)cap < 64 * nik) return -1;
    std::memcpy(out, s->christ.data(), 64 * nik * sizeof(double));
    return (long long)(64 * nik);
  }
  return -2;
}

}  // extern "C"
