// B200FemJNI.cc -- JNI glue of libb200fem.so for a Java class
// maspack.solvers.B200FemSolver (and maspack.solvers.B200FemServer), the
// neighbour of the reference's cuDSS bridge (maspack.solvers.CuDssSolver,
// CuDssSolver.java:87-163, whose glue is CuDssJNI.cc:15-747).
//
// Conventions taken from CuDssJNI.cc: the native handle is an opaque pointer
// carried as a jlong (0 = failure, message from doGetLastError); every
// method returns the library's int status (0 or a negative
// B200FEM_ERR_* code, which the Java side turns into a NumericalException as
// CuDssSolver.check does, CuDssSolver.java:289-296); Java arrays are
// borrowed for the duration of the call -- inputs released with JNI_ABORT
// (no copy back), outputs with mode 0 (copied back).  All calls are
// synchronous; a handle must not be used from two threads at once (the Java
// methods are synchronized, like CuDssSolver's).
//
// Build with a JDK:
//   g++ -O2 -shared -fPIC -I$JAVA_HOME/include -I$JAVA_HOME/include/linux
//       -I<repo>/include B200FemJNI.cc -L<repo>/artisynth_core_b200 -lb200fem
//       -o libB200FemJNI.so
// and install it where NativeLibraryManager.load finds the reference's other
// natives (lib/Linux64/lib<Name>.so.<ver>, NativeLibraryManager.java:918).
#include <jni.h>

#include "b200fem.h"

namespace {

inline b200fem_handle H(jlong h) { return reinterpret_cast<b200fem_handle>(h); }
inline b200fem_server_handle S(jlong s) { return reinterpret_cast<b200fem_server_handle>(s); }

// nodes per element of the B200FEM_ELEM_* types
int nodes_per_elem(jint type) {
  static const int n[8] = {4, 8, 6, 5, 10, 20, 15, 13};
  return (type >= 0 && type < 8) ? n[type] : 0;
}

// a borrowed double[]: released with JNI_ABORT unless marked as output
struct Doubles {
  JNIEnv* env;
  jdoubleArray arr;
  jdouble* p;
  bool out;
  Doubles(JNIEnv* e, jdoubleArray a, bool output) : env(e), arr(a), p(nullptr), out(output) {
    if (arr) p = env->GetDoubleArrayElements(arr, nullptr);
  }
  ~Doubles() {
    if (p) env->ReleaseDoubleArrayElements(arr, p, out ? 0 : JNI_ABORT);
  }
  jsize size() const { return arr ? env->GetArrayLength(arr) : 0; }
};

struct Ints {
  JNIEnv* env;
  jintArray arr;
  jint* p;
  bool out;
  Ints(JNIEnv* e, jintArray a, bool output) : env(e), arr(a), p(nullptr), out(output) {
    if (arr) p = env->GetIntArrayElements(arr, nullptr);
  }
  ~Ints() {
    if (p) env->ReleaseIntArrayElements(arr, p, out ? 0 : JNI_ABORT);
  }
  jsize size() const { return arr ? env->GetArrayLength(arr) : 0; }
};

// step parameters as a double[]: {h, alpha_m, beta_k, gx, gy, gz, tol,
// max_iter, integrator, pcg_variant, abort_on_inverted}; entries past the
// array's length keep their defaults
bool step_params(JNIEnv* env, jdoubleArray params, b200fem_step_params* sp) {
  Doubles p(env, params, false);
  const jsize n = p.size();
  if (n < 8) return false;
  *sp = {};
  sp->h = p.p[0];
  sp->alpha_m = p.p[1];
  sp->beta_k = p.p[2];
  sp->gravity[0] = p.p[3];
  sp->gravity[1] = p.p[4];
  sp->gravity[2] = p.p[5];
  sp->tol = p.p[6];
  sp->max_iter = (int)p.p[7];
  sp->integrator = n > 8 ? (int)p.p[8] : B200FEM_INTEGRATOR_BACKWARD_EULER;
  sp->pcg_variant = n > 9 ? (int)p.p[9] : 0;
  sp->abort_on_inverted = n > 10 ? (int)p.p[10] : 0;
  return true;
}

// stats as a double[]: {iterations, rel_residual, num_inverted, min_detJ, refinements}
void put_stats(JNIEnv* env, jdoubleArray stats, const b200fem_stats& st) {
  if (!stats) return;
  const jdouble out[5] = {(double)st.iterations, st.rel_residual, (double)st.num_inverted, st.min_detJ,
                          (double)st.refinements};
  jsize n = env->GetArrayLength(stats);
  env->SetDoubleArrayRegion(stats, 0, n < 5 ? n : 5, out);
}

}  // namespace

extern "C" {

// ---- handle lifecycle (CuDssJNI doInit / doDispose / doGetLastError) -----
JNIEXPORT jlong JNICALL Java_maspack_solvers_B200FemSolver_doCreate(JNIEnv*, jclass, jint device, jint precision) {
  b200fem_config cfg = {};
  cfg.device = device;
  cfg.precision = precision;
  return reinterpret_cast<jlong>(b200fem_create(&cfg));
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doDispose(JNIEnv*, jclass, jlong h) {
  return b200fem_destroy(H(h));  // idempotent, NULL accepted
}

JNIEXPORT jstring JNICALL Java_maspack_solvers_B200FemSolver_doGetLastError(JNIEnv* env, jclass, jlong h) {
  return env->NewStringUTF(b200fem_last_error(H(h)));
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doVersion(JNIEnv*, jclass) { return b200fem_version(); }

// ---- model definition ------------------------------------------------------
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSetMesh(JNIEnv* env, jclass, jlong h, jint type,
                                                                    jdoubleArray rest, jintArray conn,
                                                                    jintArray fixed) {
  const int nen = nodes_per_elem(type);
  if (!nen || !rest || !conn) return B200FEM_ERR_INVALID_ARG;
  Doubles r(env, rest, false);
  Ints c(env, conn, false);
  Ints f(env, fixed, false);
  return b200fem_set_mesh(H(h), type, r.size() / 3, r.p, c.size() / nen, c.p, f.p);
}

// a model whose elements are of several classes: types[e] per element, conn
// every element's nodes concatenated in element order
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSetMeshMixed(JNIEnv* env, jclass, jlong h,
                                                                         jintArray types, jdoubleArray rest,
                                                                         jintArray conn, jintArray fixed) {
  if (!types || !rest || !conn) return B200FEM_ERR_INVALID_ARG;
  Ints t(env, types, false);
  Doubles r(env, rest, false);
  Ints c(env, conn, false);
  Ints f(env, fixed, false);
  long long total = 0;
  for (jsize e = 0; e < t.size(); e++) {
    const int k = nodes_per_elem(t.p[e]);
    if (!k) return B200FEM_ERR_INVALID_ARG;
    total += k;
  }
  if (total != c.size()) return B200FEM_ERR_INVALID_ARG;
  return b200fem_set_mesh_mixed(H(h), r.size() / 3, r.p, t.size(), t.p, c.p, f.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSetMaterial(JNIEnv* env, jclass, jlong h, jint kind,
                                                                        jdoubleArray params, jdouble density,
                                                                        jint incomp) {
  if (!params) return B200FEM_ERR_INVALID_ARG;
  double prm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  Doubles p(env, params, false);
  for (jsize i = 0; i < p.size() && i < 8; i++) prm[i] = p.p[i];
  return b200fem_set_material(H(h), kind, prm, density, incomp);
}

// kinds[e]: B200FEM_MAT_* of element e, or B200FEM_MAT_MODEL (-1) where
// FemElement.getMaterial() is null; params: 8 per element (kinds == null
// restores the model's material everywhere)
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSetElementMaterials(JNIEnv* env, jclass, jlong h,
                                                                                jint model, jintArray kinds,
                                                                                jdoubleArray params) {
  if (!kinds) return b200fem_set_element_materials(H(h), model, 0, nullptr, nullptr);
  if (!params) return B200FEM_ERR_INVALID_ARG;
  Ints k(env, kinds, false);
  Doubles p(env, params, false);
  if ((long long)p.size() != 8LL * k.size()) return B200FEM_ERR_INVALID_ARG;
  return b200fem_set_element_materials(H(h), model, k.size(), k.p, p.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doAddModel(JNIEnv* env, jclass, jlong h, jint type,
                                                                     jdoubleArray rest, jintArray conn,
                                                                     jintArray fixed, jint kind,
                                                                     jdoubleArray params, jdouble density,
                                                                     jint incomp) {
  const int nen = nodes_per_elem(type);
  if (!nen || !rest || !conn || !params) return B200FEM_ERR_INVALID_ARG;
  double prm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  {
    Doubles p(env, params, false);
    for (jsize i = 0; i < p.size() && i < 8; i++) prm[i] = p.p[i];
  }
  Doubles r(env, rest, false);
  Ints c(env, conn, false);
  Ints f(env, fixed, false);
  int idx = -1;
  const int st = b200fem_add_model(H(h), type, r.size() / 3, r.p, c.size() / nen, c.p, f.p, kind, prm, density,
                                   incomp, &idx);
  return st == B200FEM_OK ? idx : st;  // the model's index, or the status
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doBuild(JNIEnv*, jclass, jlong h) {
  return b200fem_build(H(h));
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSetOption(JNIEnv*, jclass, jlong h, jint key,
                                                                      jint value) {
  return b200fem_set_option(H(h), key, value);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doGetOption(JNIEnv* env, jclass, jlong h, jint key,
                                                                      jintArray out) {
  int v = 0;
  const int st = b200fem_get_option(H(h), key, &v);
  if (st == B200FEM_OK && out) env->SetIntArrayRegion(out, 0, 1, &v);
  return st;
}

// ---- pattern queries (compared with createCrsBlockSlotMap) --------------
// sizes: {n_active, nnzb, crs_nnz_full, crs_nnz_upper}
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doGetSizes(JNIEnv* env, jclass, jlong h,
                                                                     jintArray sizes) {
  int s[4] = {0, 0, 0, 0};
  const int st = b200fem_get_sizes(H(h), &s[0], &s[1], &s[2], &s[3]);
  if (st == B200FEM_OK && sizes) env->SetIntArrayRegion(sizes, 0, 4, s);
  return st;
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doGetSolveIndex(JNIEnv* env, jclass, jlong h,
                                                                          jintArray sidx) {
  Ints s(env, sidx, true);
  return b200fem_get_solve_index(H(h), s.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doGetCrsIndices(JNIEnv* env, jclass, jlong h,
                                                                          jint partition, jintArray rowOffs,
                                                                          jintArray colIdxs) {
  Ints r(env, rowOffs, true);
  Ints c(env, colIdxs, true);
  return b200fem_get_crs_indices(H(h), partition, r.p, c.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doGetSlotMap(JNIEnv* env, jclass, jlong h,
                                                                       jint partition, jintArray slots) {
  Ints s(env, slots, true);
  return b200fem_get_slot_map(H(h), partition, s.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doGetMasses(JNIEnv* env, jclass, jlong h,
                                                                      jdoubleArray mass) {
  Doubles m(env, mass, true);
  return b200fem_get_masses(H(h), m.p);
}

// ---- state ---------------------------------------------------------------
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSetState(JNIEnv* env, jclass, jlong h, jdoubleArray x,
                                                                     jdoubleArray v) {
  Doubles px(env, x, false);
  Doubles pv(env, v, false);
  return b200fem_set_state(H(h), px.p, pv.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doGetState(JNIEnv* env, jclass, jlong h, jdoubleArray x,
                                                                     jdoubleArray v) {
  Doubles px(env, x, true);
  Doubles pv(env, v, true);
  return b200fem_get_state(H(h), px.p, pv.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSetExternalForces(JNIEnv* env, jclass, jlong h,
                                                                              jdoubleArray fext) {
  Doubles f(env, fext, false);
  return b200fem_set_external_forces(H(h), f.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSetPlaneConstraints(JNIEnv* env, jclass, jlong h,
                                                                                jintArray nodes,
                                                                                jdoubleArray normals,
                                                                                jdoubleArray offsets) {
  Ints n(env, nodes, false);
  Doubles q(env, normals, false);
  Doubles o(env, offsets, false);
  return b200fem_set_plane_constraints(H(h), n.size(), n.p, q.p, o.p);
}

// ---- hot path ----------------------------------------------------------------
// FemModel3d.updateStressAndStiffness: forces and the full-partition CRS
// values in the slot order of createCrsBlockSlotMap (either may be null)
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doUpdateStressStiffness(JNIEnv* env, jclass, jlong h,
                                                                                  jdoubleArray x,
                                                                                  jdoubleArray fint,
                                                                                  jdoubleArray crs) {
  Doubles px(env, x, false);
  Doubles pf(env, fint, true);
  Doubles pc(env, crs, true);
  return b200fem_update_stress_stiffness(H(h), px.p, pf.p, nullptr, pc.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doBackwardEulerStep(JNIEnv* env, jclass, jlong h,
                                                                              jdoubleArray params, jint nsteps,
                                                                              jdoubleArray stats) {
  b200fem_step_params sp;
  if (!step_params(env, params, &sp)) return B200FEM_ERR_INVALID_ARG;
  b200fem_stats st = {};
  const int status = b200fem_backward_euler_step(H(h), &sp, nsteps, &st);
  put_stats(env, stats, st);
  return status;
}

// The host keeps the state (ArtiSynth's node positions and velocities): the
// arrays are borrowed, stepped in one native call and written back.
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doBackwardEulerStepHost(JNIEnv* env, jclass, jlong h,
                                                                                  jdoubleArray params, jint nsteps,
                                                                                  jdoubleArray x, jdoubleArray v,
                                                                                  jdoubleArray stats) {
  b200fem_step_params sp;
  if (!step_params(env, params, &sp) || !x || !v) return B200FEM_ERR_INVALID_ARG;
  b200fem_stats st = {};
  int status;
  {
    Doubles px(env, x, true);
    Doubles pv(env, v, true);
    status = b200fem_backward_euler_step_host(H(h), &sp, nsteps, px.p, pv.p, &st);
  }
  put_stats(env, stats, st);
  return status;
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doMultiply(JNIEnv* env, jclass, jlong h, jdoubleArray x,
                                                                     jdoubleArray y) {
  Doubles px(env, x, false);
  Doubles py(env, y, true);
  return b200fem_spmv(H(h), px.p, py.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSolve(JNIEnv* env, jclass, jlong h, jdoubleArray b,
                                                                  jdoubleArray x, jdouble tol, jint maxIter,
                                                                  jdoubleArray stats) {
  b200fem_stats st = {};
  int status;
  {
    Doubles pb(env, b, false);
    Doubles px(env, x, true);
    status = b200fem_pcg_solve(H(h), pb.p, px.p, tol, maxIter, &st);
  }
  put_stats(env, stats, st);
  return status;
}

// Device pointers from a caller that owns its device memory (passed as
// jlong); nothing is allocated.  out: {iterations, rel_residual}
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSolveNoAlloc(JNIEnv* env, jclass, jint nRows,
                                                                         jlong rowptr, jlong col, jlong vals,
                                                                         jlong b, jlong x, jdouble tol,
                                                                         jint maxIter, jlong stream,
                                                                         jdoubleArray out) {
  int it = 0;
  double rr = 0;
  const int st = b200fem_pcg_solve_noalloc(nRows, reinterpret_cast<const int*>(rowptr),
                                           reinterpret_cast<const int*>(col), reinterpret_cast<const double*>(vals),
                                           reinterpret_cast<const double*>(b), reinterpret_cast<double*>(x), tol,
                                           maxIter, reinterpret_cast<void*>(stream), &it, &rr);
  if (out) {
    const jdouble o[2] = {(double)it, rr};
    env->SetDoubleArrayRegion(out, 0, 2, o);
  }
  return st;
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doLastTiming(JNIEnv* env, jclass, jlong h,
                                                                       jdoubleArray out) {
  double a = 0, s = 0;
  const int st = b200fem_last_timing(H(h), &a, &s);
  if (out) {
    const jdouble o[2] = {a, s};
    env->SetDoubleArrayRegion(out, 0, 2, o);
  }
  return st;
}

// ---- batched form ------------------------------------------------------------
// range: {node_offset, n_nodes, n_active}
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doModelRange(JNIEnv* env, jclass, jlong h, jint model,
                                                                       jintArray range) {
  int r[3] = {0, 0, 0};
  const int st = b200fem_model_range(H(h), model, &r[0], &r[1], &r[2]);
  if (st == B200FEM_OK && range) env->SetIntArrayRegion(range, 0, 3, r);
  return st;
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doSetActiveModels(JNIEnv* env, jclass, jlong h,
                                                                            jintArray active) {
  Ints a(env, active, false);
  return b200fem_set_active_models(H(h), a.p);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doMemoryUsage(JNIEnv* env, jclass, jlong h,
                                                                        jlongArray out) {
  unsigned long long bytes = 0;
  const int st = b200fem_memory_usage(H(h), &bytes);
  if (st == B200FEM_OK && out) {
    const jlong v = (jlong)bytes;
    env->SetLongArrayRegion(out, 0, 1, &v);
  }
  return st;
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemSolver_doGetModelStats(JNIEnv* env, jclass, jlong h,
                                                                          jintArray iterations,
                                                                          jdoubleArray residuals) {
  Ints it(env, iterations, true);
  Doubles rr(env, residuals, true);
  return b200fem_get_model_stats(H(h), it.p, rr.p);
}

// ---- served form (maspack.solvers.B200FemServer) --------------------------
// params as doStep's; budget in bytes
JNIEXPORT jlong JNICALL Java_maspack_solvers_B200FemServer_doCreate(JNIEnv* env, jclass, jint device,
                                                                    jint precision, jdouble budgetBytes,
                                                                    jint packModels, jdoubleArray params) {
  b200fem_step_params sp;
  if (!step_params(env, params, &sp)) return 0;
  b200fem_config cfg = {};
  cfg.device = device;
  cfg.precision = precision;
  return reinterpret_cast<jlong>(b200fem_server_create(&cfg, budgetBytes, packModels, &sp));
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemServer_doDispose(JNIEnv*, jclass, jlong s) {
  return b200fem_server_destroy(S(s));
}

JNIEXPORT jstring JNICALL Java_maspack_solvers_B200FemServer_doGetLastError(JNIEnv* env, jclass, jlong s) {
  return env->NewStringUTF(b200fem_server_last_error(S(s)));
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemServer_doSetOption(JNIEnv*, jclass, jlong s, jint key,
                                                                      jint value) {
  return b200fem_server_set_option(S(s), key, value);
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemServer_doAddModel(JNIEnv* env, jclass, jlong s, jint type,
                                                                     jdoubleArray rest, jintArray conn,
                                                                     jintArray fixed, jint kind,
                                                                     jdoubleArray params, jdouble density,
                                                                     jint incomp, jdoubleArray fext) {
  const int nen = nodes_per_elem(type);
  if (!nen || !rest || !conn || !params) return B200FEM_ERR_INVALID_ARG;
  double prm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  {
    Doubles p(env, params, false);
    for (jsize i = 0; i < p.size() && i < 8; i++) prm[i] = p.p[i];
  }
  Doubles r(env, rest, false);
  Ints c(env, conn, false);
  Ints f(env, fixed, false);
  Doubles fe(env, fext, false);
  int id = -1;
  const int st = b200fem_server_add_model(S(s), type, r.size() / 3, r.p, c.size() / nen, c.p, f.p, kind, prm,
                                          density, incomp, fe.p, &id);
  return st == B200FEM_OK ? id : st;
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemServer_doPreload(JNIEnv*, jclass, jlong s) {
  return b200fem_server_preload(S(s));
}

// the request's id, or the status; tArrive < 0: now
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemServer_doSubmit(JNIEnv*, jclass, jlong s, jint model,
                                                                   jint steps, jdouble tArrive) {
  int id = -1;
  const int st = b200fem_server_submit(S(s), model, steps, tArrive, &id);
  return st == B200FEM_OK ? id : st;
}

// model steps taken by this tick, or the status
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemServer_doTick(JNIEnv*, jclass, jlong s) {
  int n = 0;
  const int st = b200fem_server_tick(S(s), &n);
  return st == B200FEM_OK ? n : st;
}

// out: {state (0 queued, 1 running, 2 done, -1 failed), latency_s}
JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemServer_doPoll(JNIEnv* env, jclass, jlong s, jint request,
                                                                 jdoubleArray out) {
  int state = 0;
  double lat = 0;
  const int st = b200fem_server_poll(S(s), request, &state, &lat);
  if (st == B200FEM_OK && out) {
    const jdouble o[2] = {(double)state, lat};
    env->SetDoubleArrayRegion(out, 0, 2, o);
  }
  return st;
}

JNIEXPORT jint JNICALL Java_maspack_solvers_B200FemServer_doGetState(JNIEnv* env, jclass, jlong s, jint model,
                                                                     jdoubleArray x, jdoubleArray v) {
  Doubles px(env, x, true);
  Doubles pv(env, v, true);
  return b200fem_server_get_state(S(s), model, px.p, pv.p);
}

JNIEXPORT jdouble JNICALL Java_maspack_solvers_B200FemServer_doClock(JNIEnv*, jclass, jlong s) {
  return b200fem_server_clock(S(s));
}

}  // extern "C"
