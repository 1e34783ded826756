// -*- C++ -*-
/// @file sphere_pt.hpp
/// @brief FP32 path tracer of sphere scenes, written in the Loom kernel
/// language with Loom's own macro library (src/vm/lib/random.hpp,
/// src/vm/lib/linal.hpp).
///
/// One Loom thread traces one sample path of one pixel.  Inputs:
///   inst  instance (render request) index into the scene table
///   sid   sample index within the instance: pixel * spp + sample
/// Outputs: the radiance of the path, L0 L1 L2 (RGB, f32).
///
/// Everything an instance needs is read with the table op (b200_ops.hpp)
/// from a table of 32-bit words:
///   instance header, 16 words at inst * 16:
///     0 width  1 height  2 log2(spp)  3 seed  4 first sphere word
///     5 sphere count  6..8 camera position (f32)  9 tan(fov / 2) (f32)
///   sphere record, 8 words: centre xyz, radius, colour rgb (f32), material
///     (u32: 0 diffuse, 1 mirror, 2 glass of IOR 1.5, 3 emitter; for an
///     emitter the colour is its radiance).
/// The camera looks down -z.  Each sample is jittered in its pixel with a
/// 2x2 subpixel tent filter; paths do Russian roulette from the 5th surface
/// hit and end at the 16th.  Random numbers: Threefry-2x32 (Loom's
/// threefry2x32r32) keyed by (seed, constant), counter (pixel, sample << 20
/// | draw), turned into [0, 1) floats by gen_canonical.  The RNG is one
/// shared block ("roll") that every caller jumps to with a return index in
/// rpt, as Loom's own path-tracing kernels do (src/smallpt/vm/pt.hpp:889-914).
///
/// Ray-sphere: with oc = centre - origin and unit direction d,
/// b = oc.d, q = oc - b d, det = r^2 - q.q (computed as fms(r, r, q.q)), which
/// keeps precision for the radius-1e5 walls; the nearer root above EPS is
/// taken, branch-free.  Diffuse bounces sample the cosine-weighted
/// hemisphere by rejection-sampling a unit disk and lifting it (Malley's
/// method), so no sin/cos is needed; glass uses Fresnel-Schlick with a
/// probability split between reflection and refraction.
#pragma once

#include <vm/core.hpp>
#include <vm/lib/linal.hpp>
#include <vm/lib/random.hpp>
#include <vm/macros.hpp>
#include <vm/operators.hpp>

#include "../frontend/b200_ops.hpp"

#include <concepts>
#include <cstdint>

namespace loom::vm::b200::kernels
{
using namespace loom::vm;

// clang-format off
template <std::same_as<float> T>
KERNEL(sphere_pt, IVAR(inst), IVAR(sid))
    // ---- instance header
    IMUL(hb, inst, 16),
    TABU(w, hb),
    IADD(ti, hb, 1), TABU(h, ti),
    IADD(ti, hb, 2), TABU(sl, ti),
    IADD(ti, hb, 3), TABU(k0, ti),
    IADD(ti, hb, 4), TABU(soff, ti),
    IADD(ti, hb, 5), TABU(scnt, ti),
    IADD(ti, hb, 6), TABF(cam0, ti),
    IADD(ti, hb, 7), TABF(cam1, ti),
    IADD(ti, hb, 8), TABF(cam2, ti),
    IADD(ti, hb, 9), TABF(tanf, ti),
    // ---- pixel and sample
    IRSHFT(pix, sid, sl),
    ILSHFT(msk, 1, sl),
    ISUB(msk, msk, 1),
    IBAND(smp, sid, msk),
    IMOD(px, pix, w),
    IDIV(py, pix, w),
    // ---- RNG key and counter
    IXOR(k2, k0, 0x1bd11bda),
    IXOR(k2, k2, 0x9e3779b9),
    IMOV(c0, pix),
    ILSHFT(c1, smp, 20),
    IMOV(rpt, 0),
    JMP(roll),

    // ---- primary ray
    LABEL(prim),
    IBAND(sub, smp, 3),
    IBAND(sbx, sub, 1),
    IRSHFT(sby, sub, 1),
    // tent filter: r < 1 ? sqrt(r) - 1 : 1 - sqrt(2 - r), r = 2u
    TMUL(ra, u0, 2),
    TSQRT(fa, ra), TSUB(fa, fa, 1),
    TSUB(fb, 2, ra), TSQRT(fb, fb), TSUB(fb, 1, fb),
    TLT(cnd, ra, 1),
    TCMOV(fdx, cnd, fa, fb),
    TMUL(ra, u1, 2),
    TSQRT(fa, ra), TSUB(fa, fa, 1),
    TSUB(fb, 2, ra), TSQRT(fb, fb), TSUB(fb, 1, fb),
    TLT(cnd, ra, 1),
    TCMOV(fdy, cnd, fa, fb),
    // position on the image plane in pixels
    MOV(TVAR(fx), IVAR(sbx)),
    TADD(fx, fx, 0.5), TADD(fx, fx, fdx), TMUL(fx, fx, 0.5),
    MOV(TVAR(fp), IVAR(px)), TADD(fx, fx, fp),
    MOV(TVAR(fy), IVAR(sby)),
    TADD(fy, fy, 0.5), TADD(fy, fy, fdy), TMUL(fy, fy, 0.5),
    MOV(TVAR(fp), IVAR(py)), TADD(fy, fy, fp),
    // camera direction
    MOV(TVAR(fw), IVAR(w)), MOV(TVAR(fh), IVAR(h)),
    TDIV(fx, fx, fw), TMUL(fx, fx, 2), TSUB(fx, fx, 1),
    TDIV(asp, fw, fh), TMUL(fx, fx, asp), TMUL(d0, fx, tanf),
    TDIV(fy, fy, fh), TMUL(fy, fy, 2), TSUB(fy, 1, fy), TMUL(d1, fy, tanf),
    TMOV(d2, -1),
    INSERT_TMACRO(vec3_norm, CS(d), CS(tmp)),
    TMOV(o0, cam0), TMOV(o1, cam1), TMOV(o2, cam2),
    TMOV(T0, 1), TMOV(T1, 1), TMOV(T2, 1),
    TMOV(L0, 0), TMOV(L1, 0), TMOV(L2, 0),
    IMOV(depth, 0),

    // ---- nearest sphere along the ray
    LABEL(bounce),
    TMOV(tmin, 1e30),
    IMOV(hid, scnt),
    IMOV(i, 0),
    IMOV(sp, soff),
    LABEL(isect),
    TABF(s0, sp), IADD(ti, sp, 1), TABF(s1, ti),
    IADD(ti, sp, 2), TABF(s2, ti), IADD(ti, sp, 3), TABF(sr, ti),
    TSUB(oc0, s0, o0), TSUB(oc1, s1, o1), TSUB(oc2, s2, o2),
    INSERT_TMACRO(vec3_dot, CS(bq), CS(oc), CS(d)),
    TNEG(nbq, bq),
    TFMA(q0, nbq, d0, oc0), TFMA(q1, nbq, d1, oc1), TFMA(q2, nbq, d2, oc2),
    INSERT_TMACRO(vec3_dot, CS(l2), CS(q), CS(q)),
    TFMS(det, sr, sr, l2),
    TGE(hit, det, 0),
    TMAX(det, det, 0),
    TSQRT(sq, det),
    TSUB(t0, bq, sq), TADD(t1, bq, sq),
    TGT(cnd, t0, 0.05),
    TCMOV(tt, cnd, t0, t1),
    TANDGT(hit, hit, tt, 0.05),
    TANDLT(hit, hit, tt, tmin),
    TCMOV(tmin, hit, tt, tmin),
    ICMOV(hid, hit, i, hid),
    IADD(i, i, 1), IADD(sp, sp, 8),
    ILT(cnd, i, scnt),
    IPJMP2(cnd, shade, isect),

    LABEL(shade),
    IGE(cnd, hid, scnt),
    IPJMP2(cnd, hitp, HALT),
    LABEL(hitp),
    IMUL(sp, hid, 8), IADD(sp, sp, soff),
    TABF(s0, sp), IADD(ti, sp, 1), TABF(s1, ti),
    IADD(ti, sp, 2), TABF(s2, ti), IADD(ti, sp, 3), TABF(sr, ti),
    IADD(ti, sp, 4), TABF(cr, ti), IADD(ti, sp, 5), TABF(cg, ti),
    IADD(ti, sp, 6), TABF(cb, ti), IADD(ti, sp, 7), TABU(mat, ti),
    TFMA(x0, d0, tmin, o0), TFMA(x1, d1, tmin, o1), TFMA(x2, d2, tmin, o2),
    TSUB(n0, x0, s0), TSUB(n1, x1, s1), TSUB(n2, x2, s2),
    TDIV(n0, n0, sr), TDIV(n1, n1, sr), TDIV(n2, n2, sr),
    IEQ(cnd, mat, 3),
    IPJMP2(cnd, surf, emit),
    LABEL(emit),
    TFMA(L0, T0, cr, L0), TFMA(L1, T1, cg, L1), TFMA(L2, T2, cb, L2),
    JMP(HALT),

    // ---- path length: at most 16 surface hits, Russian roulette from the 5th
    LABEL(surf),
    IADD(depth, depth, 1),
    IGE(cnd, depth, 16),
    IPJMP2(cnd, rrchk, HALT),
    LABEL(rrchk),
    IGE(cnd, depth, 5),
    IPJMP2(cnd, scatter, rr_roll),
    LABEL(rr_roll),
    IMOV(rpt, 1),
    JMP(roll),
    LABEL(rr),
    TMAX(p, cr, cg), TMAX(p, p, cb),
    TLT(cnd, u0, p),
    IPJMP2(cnd, HALT, rr_keep),
    LABEL(rr_keep),
    TDIV(cr, cr, p), TDIV(cg, cg, p), TDIV(cb, cb, p),

    LABEL(scatter),
    TMUL(T0, T0, cr), TMUL(T1, T1, cg), TMUL(T2, T2, cb),
    TMOV(o0, x0), TMOV(o1, x1), TMOV(o2, x2),
    INSERT_TMACRO(vec3_dot, CS(dn), CS(n), CS(d)),
    TLT(into, dn, 0),
    TNEG(m0, n0), TNEG(m1, n1), TNEG(m2, n2),
    TCMOV(nl0, into, n0, m0), TCMOV(nl1, into, n1, m1), TCMOV(nl2, into, n2, m2),
    IPJMP3(mat, diffuse, mirror, glass),

    // ---- specular reflection: d <- d - 2 (n.d) n
    LABEL(mirror),
    TMUL(dn2, dn, -2),
    TFMA(d0, dn2, n0, d0), TFMA(d1, dn2, n1, d1), TFMA(d2, dn2, n2, d2),
    JMP(bounce),

    // ---- diffuse: cosine-weighted hemisphere around nl
    LABEL(diffuse),
    TABS(aw, nl0), TGT(cnd, aw, 0.1),
    TCMOV(a0, cnd, 0, 1), TCMOV(a1, cnd, 1, 0), TMOV(a2, 0),
    INSERT_TMACRO(vec3_cross, CS(uu), CS(a), CS(nl), CS(tmp)),
    INSERT_TMACRO(vec3_norm, CS(uu), CS(tmp)),
    INSERT_TMACRO(vec3_cross, CS(vv), CS(nl), CS(uu), CS(tmp)),
    LABEL(disk_roll),
    IMOV(rpt, 2),
    JMP(roll),
    LABEL(disk),
    TMUL(dx, u0, 2), TSUB(dx, dx, 1),
    TMUL(dy, u1, 2), TSUB(dy, dy, 1),
    TMUL(rr2, dx, dx), TFMA(rr2, dy, dy, rr2),
    TLT(cnd, rr2, 1),
    IPJMP2(cnd, disk_roll, disk_ok),
    LABEL(disk_ok),
    TSUB(dz, 1, rr2), TSQRT(dz, dz),
    TMUL(d0, uu0, dx), TFMA(d0, vv0, dy, d0), TFMA(d0, nl0, dz, d0),
    TMUL(d1, uu1, dx), TFMA(d1, vv1, dy, d1), TFMA(d1, nl1, dz, d1),
    TMUL(d2, uu2, dx), TFMA(d2, vv2, dy, d2), TFMA(d2, nl2, dz, d2),
    INSERT_TMACRO(vec3_norm, CS(d), CS(tmp)),
    JMP(bounce),

    // ---- glass (IOR 1.5): Fresnel-Schlick split between reflection and refraction
    LABEL(glass),
    TDIV(nin, 1, 1.5),
    TCMOV(nnt, into, nin, 1.5),
    INSERT_TMACRO(vec3_dot, CS(ddn), CS(d), CS(nl)),
    TMUL(c2, ddn, ddn), TSUB(c2, 1, c2),
    TMUL(nn2, nnt, nnt), TMUL(c2, c2, nn2), TSUB(c2, 1, c2),
    TLT(cnd, c2, 0),
    IPJMP2(cnd, refr, mirror),
    LABEL(refr),
    TSQRT(sc, c2), TFMA(sc, ddn, nnt, sc),
    TNEG(nsc, sc), TCMOV(sc, into, sc, nsc),
    TNEG(nsc, sc),
    TMUL(td0, d0, nnt), TFMA(td0, nsc, n0, td0),
    TMUL(td1, d1, nnt), TFMA(td1, nsc, n1, td1),
    TMUL(td2, d2, nnt), TFMA(td2, nsc, n2, td2),
    INSERT_TMACRO(vec3_norm, CS(td), CS(tmp)),
    TDIV(r0, 0.5, 2.5), TMUL(r0, r0, r0),
    INSERT_TMACRO(vec3_dot, CS(ctn), CS(td), CS(n)),
    TNEG(nddn, ddn), TCMOV(cc, into, nddn, ctn), TSUB(cc, 1, cc),
    TMUL(c5, cc, cc), TMUL(c5, c5, c5), TMUL(c5, c5, cc),
    TSUB(re, 1, r0), TFMA(re, re, c5, r0),
    TSUB(tr, 1, re),
    TFMA(pp, re, 0.5, 0.25),
    TDIV(rp, re, pp), TSUB(tp, 1, pp), TDIV(tp, tr, tp),
    IMOV(rpt, 3),
    JMP(roll),
    LABEL(fres),
    TLT(cnd, u0, pp),
    IPJMP2(cnd, take_refr, take_refl),
    LABEL(take_refl),
    TMUL(T0, T0, rp), TMUL(T1, T1, rp), TMUL(T2, T2, rp),
    JMP(mirror),
    LABEL(take_refr),
    TMUL(T0, T0, tp), TMUL(T1, T1, tp), TMUL(T2, T2, tp),
    TMOV(d0, td0), TMOV(d1, td1), TMOV(d2, td2),
    JMP(bounce),

    // ---- shared RNG: two uniforms in u0, u1, then back to the caller
    LABEL(roll),
    IMOV(u0, c0), IMOV(u1, c1),
    INSERT_MACRO(threefry2x32r32, CS(u0), CS(u1), CS(k0), CS(0x9e3779b9), CS(k2), CS(tmp1), CS(tmp2)),
    IADD(c1, c1, 1),
    INSERT_TMACRO(gen_canonical, CS(u0)),
    INSERT_TMACRO(gen_canonical, CS(u1)),
    IPJMP4(rpt, prim, rr, disk, fres)
KERNEL_END(TVAR(L0), TVAR(L1), TVAR(L2));
// clang-format on
} // namespace loom::vm::b200::kernels
