// ffvils_gpu_parity.cpp -- the pressure solve driven from C++ the way
// FFV-HC's Solver::UpdateP drives FFVILS (src/FFV/Solver.cpp:5294-5688),
// through FFVILSGpu and the C ABI, checked bit for bit against the CPU
// oracle (linked for the comparison only).
//
// Steps: synthetic sphere grid -> exchange u (P02) -> bcut_calc_ab_p (P03)
// -> fold outer BCs (P05) -> RBGS -> CG -> BiCGSTAB -> exchange p (P07).
// Exit status 0 when every residual and every pressure value is identical.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../ffv-hc_b200/host/FFVILSGpu.h"
#include "../../include/ffvgpu.h"

extern "C" {
struct Oracle;
Oracle* orc_create(int nb, int n, int g, const int* level, const long* idx3,
                   const double* dom_org, double root_len, const int* root_grid);
void orc_destroy(Oracle*);
double* orc_field(Oracle*, int id);
int* orc_ifield(Oracle*, int id);
void orc_set_threads(Oracle*, int);
void orc_set_reduction(Oracle*, int);
void orc_set_bc(Oracle*, const int* type6, const double* value6);
void orc_exchange(Oracle*, int fid, const int* type6, const double* value6);
void orc_assemble_p(Oracle*, double rhof, double dt);
void orc_fold_bc(Oracle*);
int orc_rbgs(Oracle*, double omega, int countMax, double eps, int* count, double* residual,
             double* hist);
int orc_cg(Oracle*, double omega, int countPre, int countMax, double eps, int* count,
           double* residual, double* hist);
int orc_bicgstab(Oracle*, double omega, int countPre, int countMax, double eps, int* count,
                 double* residual, double* hist);
}

static int fail(const char* what) {
  std::printf("FAIL %s: %s\n", what, ffvgpu_last_error());
  return 1;
}

int main(int argc, char** argv) {
  const int level = argc > 1 ? std::atoi(argv[1]) : 2;
  ffvgpu_sphere_params sp = {{-4.0, -4.0, -4.0}, {4, 2, 2}, 4.0, level, {0.0, 0.0, 0.0}, 0.5, 0.5};
  ffvgpu_sphere_grid* sg = nullptr;
  if (ffvgpu_sphere_grid_create(&sp, &sg) != FFVGPU_OK) return fail("sphere grid");
  const int nb = ffvgpu_sphere_grid_num_blocks(sg);
  std::vector<int32_t> lev(nb), idx(3 * nb);
  ffvgpu_sphere_grid_blocks(sg, lev.data(), idx.data());
  const int vc = 2, w = 16 + 2 * vc;
  const size_t n = (size_t)nb * w * w * w;
  std::vector<double> ux(n), uy(n), uz(n), c[6];
  std::vector<int32_t> cid[6], pid(n);
  double* cp[6];
  int32_t* ip[6];
  for (int f = 0; f < 6; ++f) {
    c[f].resize(n);
    cid[f].resize(n);
    cp[f] = c[f].data();
    ip[f] = cid[f].data();
  }
  if (ffvgpu_sphere_grid_fill(sg, 7, 0.01, vc, ux.data(), uy.data(), uz.data(), cp, ip,
                              pid.data()) != FFVGPU_OK)
    return fail("fill");

  // pressure BCs of examples/FlowPastASphere/sphere.tpp; velocity inlet (1,0,0)
  const int pt[6] = {FFVGPU_BC_NEUMANN, FFVGPU_BC_DIRICHLET, FFVGPU_BC_NEUMANN,
                     FFVGPU_BC_NEUMANN, FFVGPU_BC_NEUMANN, FFVGPU_BC_NEUMANN};
  const double pv[6] = {0, 0, 0, 0, 0, 0};
  const int ut[6] = {FFVGPU_BC_DIRICHLET, FFVGPU_BC_NEUMANN, FFVGPU_BC_NEUMANN,
                     FFVGPU_BC_NEUMANN, FFVGPU_BC_NEUMANN, FFVGPU_BC_NEUMANN};
  const double uv[3][6] = {{1, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0}};

  ffvgpu_grid_desc d;
  std::memset(&d, 0, sizeof(d));
  d.num_blocks = nb;
  d.cells = 16;
  d.level = lev.data();
  d.block_index = idx.data();
  d.domain_origin[0] = d.domain_origin[1] = d.domain_origin[2] = -4.0;
  d.root_length = 4.0;
  d.root_grid[0] = 4;
  d.root_grid[1] = 2;
  d.root_grid[2] = 2;
  for (int f = 0; f < 6; ++f) {
    d.bc_type[f] = pt[f];
    d.bc_value[f] = pv[f];
  }
  ffvgpu_pool* pool = nullptr;
  if (ffvgpu_pool_create(&d, &pool) != FFVGPU_OK) return fail("pool");
  const ffvgpu_field uf[3] = {FFVGPU_FIELD_UX, FFVGPU_FIELD_UY, FFVGPU_FIELD_UZ};
  const double* uh[3] = {ux.data(), uy.data(), uz.data()};
  for (int q = 0; q < 3; ++q)
    if (ffvgpu_pool_upload(pool, uf[q], uh[q], vc) != FFVGPU_OK) return fail("upload u");
  for (int f = 0; f < 6; ++f) {
    if (ffvgpu_pool_upload(pool, (ffvgpu_field)(FFVGPU_FIELD_C0 + f), cp[f], vc) != FFVGPU_OK ||
        ffvgpu_pool_upload(pool, (ffvgpu_field)(FFVGPU_IFIELD_CID0 + f), ip[f], vc) != FFVGPU_OK)
      return fail("upload cut");
  }
  if (ffvgpu_pool_upload(pool, FFVGPU_IFIELD_PID, pid.data(), vc) != FFVGPU_OK)
    return fail("upload pid");
  for (int q = 0; q < 3; ++q)
    if (ffvgpu_exchange(pool, uf[q], ut, uv[q]) != FFVGPU_OK) return fail("exchange u");
  if (ffvgpu_assemble_p(pool, 1.0, 0.002) != FFVGPU_OK) return fail("assemble");
  if (ffvgpu_fold_bc(pool) != FFVGPU_OK) return fail("fold");
  if (ffvgpu_fill(pool, FFVGPU_FIELD_X, 0.0) != FFVGPU_OK) return fail("fill x");

  // the same steps in the oracle
  std::vector<long> idxl(idx.begin(), idx.end());
  const double org[3] = {-4.0, -4.0, -4.0};
  const int rg[3] = {4, 2, 2};
  Oracle* O = orc_create(nb, 16, vc, lev.data(), idxl.data(), org, 4.0, rg);
  orc_set_threads(O, 8);
  orc_set_reduction(O, 1);
  orc_set_bc(O, pt, pv);
  std::memcpy(orc_field(O, 9), ux.data(), n * 8);
  std::memcpy(orc_field(O, 10), uy.data(), n * 8);
  std::memcpy(orc_field(O, 11), uz.data(), n * 8);
  for (int f = 0; f < 6; ++f) {
    std::memcpy(orc_field(O, 12 + f), cp[f], n * 8);
    std::memcpy(orc_ifield(O, f), ip[f], n * 4);
  }
  std::memcpy(orc_ifield(O, 6), pid.data(), n * 4);
  for (int q = 0; q < 3; ++q) orc_exchange(O, 9 + q, ut, uv[q]);
  orc_assemble_p(O, 1.0, 0.002);
  orc_fold_bc(O);

  FFVILSGpu ils(false);
  const int sweeps = 60, cgmax = 25;
  std::vector<double> hg(sweeps), ho(sweeps), cg_g(cgmax), cg_o(cgmax);
  int count = 0, ocount = 0;
  double residual = 0, oresidual = 0;
  ils.RBGS(pool, 1.5, sweeps, 0.0, count, residual, hg.data());
  orc_rbgs(O, 1.5, sweeps, 0.0, &ocount, &oresidual, ho.data());
  int bad = 0;
  if (count != ocount || residual != oresidual) bad++;
  for (int i = 0; i < sweeps; ++i) bad += hg[i] != ho[i];
  ils.CG(pool, 1.0, 2, cgmax, 1e-10, count, residual, cg_g.data());
  orc_cg(O, 1.0, 2, cgmax, 1e-10, &ocount, &oresidual, cg_o.data());
  if (count != ocount || residual != oresidual) bad++;
  const int nh = (count >= 1 && count <= cgmax) ? count : cgmax;
  for (int i = 0; i < nh; ++i) bad += cg_g[i] != cg_o[i];
  // then the reference's default solver from the current x
  std::vector<double> bi_g(cgmax), bi_o(cgmax);
  ils.BiCGSTAB(pool, 1.0, 2, cgmax, 1e-12, count, residual, bi_g.data());
  orc_bicgstab(O, 1.0, 2, cgmax, 1e-12, &ocount, &oresidual, bi_o.data());
  if (count != ocount || residual != oresidual) bad++;
  const int nb2 = (count >= 1 && count <= cgmax) ? count : cgmax;
  for (int i = 0; i < nb2; ++i) bad += bi_g[i] != bi_o[i];
  std::vector<double> p(n);
  if (ffvgpu_pool_download(pool, FFVGPU_FIELD_X, p.data(), vc) != FFVGPU_OK) return fail("download");
  const double* po = orc_field(O, 0);
  long diff = 0;
  for (int b = 0; b < nb; ++b)
    for (int k = 0; k < 16; ++k)
      for (int j = 0; j < 16; ++j)
        for (int i = 0; i < 16; ++i) {
          const size_t m = (size_t)b * w * w * w + (i + vc) + w * ((j + vc) + (size_t)w * (k + vc));
          diff += p[m] != po[m];
        }
  std::printf("blocks %d rbgs residual %.17g cg count %d residual %.17g mismatches %d/%ld\n", nb,
              hg[sweeps - 1], count, residual, bad, diff);
  orc_destroy(O);
  ffvgpu_pool_destroy(pool);
  ffvgpu_sphere_grid_destroy(sg);
  return (bad || diff) ? 1 : 0;
}
