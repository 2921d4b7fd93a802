// The tangent-linear run of a creature's trial (included by adjoint.cu,
// inside its namespace, after Backward): the forward derivative of the
// fitness along a direction of the start positions, the muscles' record
// fields, the nodes' friction and the nodes' masses, carried substep by
// substep beside the FP32 trajectory itself.
//
// Each substep first takes the derivative of the muscle pass from the
// substep's start state, then runs the forward substep through
// Backward::substep_kept (so the trajectory and every contact, slip and
// joint-limit mode are those of the creature kernel, to the bit), then the
// derivative of each later pass in the forward order from the values that
// pass saw (the kept lines). Every pass here is the transpose of the
// backward run's reverse pass, so for a direction u <adjoint gradient, u>
// equals the tangent's d fitness up to the rounding of
// the two FP32 derivative computations: a check of the adjoint that does not
// depend on a second trajectory (an FP64 tangent takes its own contact
// modes). The worlds of the gradients: calm, and the effects worlds with or
// without tremors (no mud, brambles or gaps).
template <class W, int RATE>
struct Tangent {
    using B = Backward<W, RATE>;
    using Body = typename B::Body;
    using C = Clock<RATE>;
    const B& bw;
    const NodeTables& d;  // tangents: positions, velocities, muscle forces then start positions, (energy, demand)
    // The creature's parameter directions: 9 floats a muscle slot in the
    // gradient's order (amplitude, hill, cap, 1/capacity, phase, duty,
    // 1/duty, 1/(1-duty), stiffness), one friction a node row; null for 0.
    const float* du_muscle;
    const float* du_friction;
    const float* du_mass;  // one mass a node row; null for 0

    // The tangents of node i's mass and inverse mass.
    __device__ __forceinline__ float dmass(unsigned i) const { return du_mass ? du_mass[i] : 0.0f; }
    __device__ __forceinline__ float dinv(unsigned i, float im) const { return -im * im * dmass(i); }

    __device__ __forceinline__ float mu_dir(unsigned k, unsigned f) const {
        return du_muscle ? du_muscle[kGradMuscle * k + f] : 0.0f;
    }

    // Tangent of the step's demands (Creature::muscle_demands; the
    // transpose of Backward::demands_back) into d.muscle().y.
    __device__ __forceinline__ void demands_tan(float t_now) const {
        const Body& b = bw.b;
        const LaneRegs& r = b.r;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        for (unsigned k = 0u; k < r.muscles; k++) {
            const unsigned m0 = S.muscle + 5u * k;
            const float4 r0 = L.get_cold(m0 + kRhythm0), r1 = L.get_cold(m0 + kRhythm1);
            const float offset = L.word_cold(m0 + kMState, 2);
            const float before = rhythm(t_now, r0.y, r0.z, offset, r0.w, r1.x, r1.y);
            const float after = rhythm(t_now + C::dt, r0.y, r0.z, offset, r0.w, r1.x, r1.y);
            const float shortening = r0.x * (after - before) * C::rate;
            const float xd = shortening * r1.z * 0.25f;
            float dd = 0.0f;
            if (!r.limp && xd >= 0.0f && du_muscle) {
                float4 ga = make_float4(0.0f, 0.0f, 0.0f, 0.0f), gb = ga;
                B::rhythm_back(t_now + C::dt, r0, r1, offset, 1.0f, ga);
                B::rhythm_back(t_now, r0, r1, offset, 1.0f, gb);
                const float da = ga.x * mu_dir(k, 4) + ga.y * mu_dir(k, 5) + ga.z * mu_dir(k, 6) + ga.w * mu_dir(k, 7);
                const float db = gb.x * mu_dir(k, 4) + gb.y * mu_dir(k, 5) + gb.z * mu_dir(k, 6) + gb.w * mu_dir(k, 7);
                const float dshort = (mu_dir(k, 0) * (after - before) + r0.x * (da - db)) * C::rate;
                dd = (dshort * r1.z + shortening * mu_dir(k, 8)) * 0.25f;
            }
            d.muscle(k).y = dd;
        }
    }

    // Tangent of the muscle pass (Creature::muscle_forces) from the start
    // state in the tables: the muscle forces' tangents into d.f and the new
    // energy stores' into d.muscle().x.
    __device__ __forceinline__ void muscles_tan() const {
        const Body& b = bw.b;
        const LaneRegs& r = b.r;
        const NodeTables& t = b.t;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const ce_params& p = b.p;
        const float c = kMuscleRecovery * p.muscle_recovery * C::h;
        for (unsigned i = 0u; i < r.nodes; i++) {
            d.f(i) = make_float2(0.0f, 0.0f);
        }
        for (unsigned k = 0u; k < r.muscles; k++) {
            const unsigned m0 = S.muscle + 5u * k;
            const float4 q0 = L.get(m0 + kPull0), q1 = L.get(m0 + kPull1);
            const float2 ms = t.muscle(k);
            const unsigned nodes = __float_as_uint(q0.x);
            const unsigned a0 = nodes & 255u, a1 = (nodes >> 8u) & 255u, b0 = (nodes >> 16u) & 255u,
                           b1 = nodes >> 24u;
            const float anchor_a = q0.y, anchor_b = q0.z, hill = q0.w;
            const float cap = q1.x, inv_capacity = q1.y, tendon_k = q1.z, slack = q1.w;
            const float4 A0 = t.at(a0), A1 = t.at(a1), B0 = t.at(b0), B1 = t.at(b1);
            const float2 dA0 = d.pos(a0), dA1 = d.pos(a1), dB0 = d.pos(b0), dB1 = d.pos(b1);
            const float2 vA0 = d.vel(a0), vA1 = d.vel(a1), vB0 = d.vel(b0), vB1 = d.vel(b1);
            const float ax = A0.x + (A1.x - A0.x) * anchor_a, ay = A0.y + (A1.y - A0.y) * anchor_a;
            const float avx = A0.z + (A1.z - A0.z) * anchor_a, avy = A0.w + (A1.w - A0.w) * anchor_a;
            const float bx = B0.x + (B1.x - B0.x) * anchor_b, by = B0.y + (B1.y - B0.y) * anchor_b;
            const float bvx = B0.z + (B1.z - B0.z) * anchor_b, bvy = B0.w + (B1.w - B0.w) * anchor_b;
            const float2 dpa = make_float2(dA0.x + (dA1.x - dA0.x) * anchor_a, dA0.y + (dA1.y - dA0.y) * anchor_a);
            const float2 dva = make_float2(vA0.x + (vA1.x - vA0.x) * anchor_a, vA0.y + (vA1.y - vA0.y) * anchor_a);
            const float2 dpb = make_float2(dB0.x + (dB1.x - dB0.x) * anchor_b, dB0.y + (dB1.y - dB0.y) * anchor_b);
            const float2 dvb = make_float2(vB0.x + (vB1.x - vB0.x) * anchor_b, vB0.y + (vB1.y - vB0.y) * anchor_b);
            const float dx = bx - ax, dy = by - ay;
            const float ddx = dpb.x - dpa.x, ddy = dpb.y - dpa.y;
            const float len0 = sqrtf(dx * dx + dy * dy);
            const float len = fmaxf(len0, 1e-6f);
            const float dlen = len0 >= 1e-6f ? (dx * ddx + dy * ddy) / len : 0.0f;
            const float ex = dx / len, ey = dy / len;
            const float dex = (ddx - ex * dlen) / len, dey = (ddy - ey * dlen) / len;
            const float rvx = bvx - avx, rvy = bvy - avy;
            const float drvx = dvb.x - dva.x, drvy = dvb.y - dva.y;
            const float lengthening = rvx * ex + rvy * ey;
            const float dlg = drvx * ex + rvx * dex + drvy * ey + rvy * dey;
            const float dhill = mu_dir(k, 1), dcap = mu_dir(k, 2), dicap = mu_dir(k, 3);
            const float drive0 = ms.y * ms.x, ddrive0 = ms.y * d.muscle(k).x + d.muscle(k).y * ms.x;
            float drive = drive0, ddrive = ddrive0;
            if (hill > 0.0f) {
                const float hz = 1.0f + lengthening * hill;
                const float hc = clampf(hz, 0.0f, 1.0f);
                drive = drive0 * hc;
                ddrive = ddrive0 * hc +
                         ((hz >= 0.0f && hz <= 1.0f) ? drive0 * (dlg * hill + lengthening * dhill) : 0.0f);
            }
            const float ya = drive + lengthening * 0.15f;
            const float dactive = (ya >= -cap && ya <= cap) ? ddrive + 0.15f * dlg : (ya > cap ? dcap : -dcap);
            const float active = clampf(ya, -cap, cap);
            const float m1 = fminf(drive, cap), m2 = fmaxf(-lengthening, 0.0f);
            const float dm1 = drive <= cap ? ddrive : dcap, dm2 = -lengthening >= 0.0f ? -dlg : 0.0f;
            const float work = m1 * m2 * C::h, dwork = (dm1 * m2 + m1 * dm2) * C::h;
            const float z = ms.x - work * inv_capacity * p.inv_muscle_energy + c * (1.0f - ms.x);
            const float dz = d.muscle(k).x * (1.0f - c) -
                             (dwork * inv_capacity + work * dicap) * p.inv_muscle_energy;
            d.muscle(k).x = (z >= 0.0f && z <= 1.0f) ? dz : 0.0f;
            const float pull = active + tendon_k * fmaxf(len - slack, 0.0f);
            const float dpull = dactive + (len - slack >= 0.0f ? tendon_k * dlen : 0.0f);
            const float dfx = dex * pull + ex * dpull, dfy = dey * pull + ey * dpull;
            float2 e = d.f(a0);
            d.f(a0) = make_float2(e.x + dfx * (1.0f - anchor_a), e.y + dfy * (1.0f - anchor_a));
            e = d.f(a1);
            d.f(a1) = make_float2(e.x + dfx * anchor_a, e.y + dfy * anchor_a);
            e = d.f(b0);
            d.f(b0) = make_float2(e.x - dfx * (1.0f - anchor_b), e.y - dfy * (1.0f - anchor_b));
            e = d.f(b1);
            d.f(b1) = make_float2(e.x - dfx * anchor_b, e.y - dfy * anchor_b);
        }
    }

    // Tangent of the air and water drag on the bones (Creature::drag_item),
    // bone by bone as the pass runs, from the velocities each bone saw
    // (A.drag); the water's wet share and the bone's direction come from the
    // substep's start positions (the forward force table holds them, d.pos
    // still their tangents: the integration's tangent comes after).
    __device__ __forceinline__ void drag_tan() const {
        const Body& b = bw.b;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const ce_params& p = b.p;
        const unsigned bones = b.r.nodes - 1u;
        for (unsigned j = 0u; j < bones; j++) {
            const float4 ba = L.get(S.bone + 2u * j), bb = L.get(S.bone + 2u * j + 1u);
            const float4 pre = L.get(bw.A.drag + j);
            const unsigned i0 = __float_as_uint(ba.x), i1 = j + 1u;
            const float wx = 0.5f * (pre.x + pre.z), wy = 0.5f * (pre.y + pre.w);
            const float speed = sqrtf(wx * wx + wy * wy);
            const float limit = bb.y;
            const float k_air = fminf(bb.x * speed, limit);
            const float2 l0 = d.vel(i0), l1 = d.vel(i1);
            const float dwx = 0.5f * (l0.x + l1.x), dwy = 0.5f * (l0.y + l1.y);
            const float dspeed = speed > 0.0f ? (wx * dwx + wy * dwy) / speed : 0.0f;
            const float dlimit = du_mass ? 0.5f * C::inv_h * (dmass(i0) + dmass(i1)) : 0.0f;
            const float dk = bb.x * speed <= limit ? bb.x * dspeed : dlimit;
            float dfx = -wx * k_air, dfy = -wy * k_air;
            float ddfx = -(dwx * k_air + wx * dk), ddfy = -(dwy * k_air + wy * dk);
            if (b.w.has(CE_FLAG_WATER)) {
                const float r0 = L.get(S.node + i0).z, r1 = L.get(S.node + i1).z;
                const float width = r0 + r1;
                const float2 p0 = b.t.f(i0), p1 = b.t.f(i1), dp0 = d.pos(i0), dp1 = d.pos(i1);
                const float z0 = (p.water - (p0.y - r0)) / (2.0f * r0);
                const float z1 = (p.water - (p1.y - r1)) / (2.0f * r1);
                const float wet = 0.5f * (clampf(z0, 0.0f, 1.0f) + clampf(z1, 0.0f, 1.0f));
                const float dwet = 0.5f * ((z0 >= 0.0f && z0 <= 1.0f ? -dp0.y / (2.0f * r0) : 0.0f) +
                                           (z1 >= 0.0f && z1 <= 1.0f ? -dp1.y / (2.0f * r1) : 0.0f));
                const float ax = (p1.x - p0.x) / ba.y, ay = (p1.y - p0.y) / ba.y;
                const float dax = (dp1.x - dp0.x) / ba.y, day = (dp1.y - dp0.y) / ba.y;
                const float along = wx * ax + wy * ay;
                const float dalong = dwx * ax + dwy * ay + wx * dax + wy * day;
                const float lx = ax * along, ly = ay * along;
                const float dlx = dax * along + ax * dalong, dly = day * along + ay * dalong;
                const float sx = wx - lx, sy = wy - ly, dsx = dwx - dlx, dsy = dwy - dly;
                const float xw = kWaterDrag * wet * ba.y * width * speed;
                const float k_water = fminf(xw, limit);
                const float dkw = xw <= limit ? kWaterDrag * ba.y * width * (dwet * speed + wet * dspeed) : dlimit;
                dfx -= sx * k_water + lx * k_water * kWaterAlong;
                dfy -= sy * k_water + ly * k_water * kWaterAlong;
                ddfx -= dsx * k_water + sx * dkw + kWaterAlong * (dlx * k_water + lx * dkw);
                ddfy -= dsy * k_water + sy * dkw + kWaterAlong * (dly * k_water + ly * dkw);
            }
            float ds0 = 0.0f, ds1 = 0.0f;
            if (du_mass) {
                ds0 = 0.5f * C::h * dinv(i0, L.get(S.node + i0).y);
                ds1 = 0.5f * C::h * dinv(i1, L.get(S.node + i1).y);
            }
            d.vel(i0) = make_float2(l0.x + bb.z * ddfx + ds0 * dfx, l0.y + bb.z * ddfy + ds0 * dfy);
            d.vel(i1) = make_float2(l1.x + bb.w * ddfx + ds1 * dfx, l1.y + bb.w * ddfy + ds1 * dfy);
        }
    }

    // Tangent of the integration (Creature::integrate_item): of the world
    // forces (gravity, wind, buoyancy) only the buoyancy moves with the state,
    // through the wet share of the start height; d.f takes the start
    // positions' tangents.
    __device__ __forceinline__ void integrate_tan() const {
        const Body& b = bw.b;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const ce_params& p = b.p;
        for (unsigned i = 0u; i < b.r.nodes; i++) {
            const float4 nr = L.get(S.node + i);
            const float im = nr.y;
            const float2 dp = d.pos(i), dfp = d.f(i);
            float dfy = 0.0f;
            if (b.w.has(CE_FLAG_WATER)) {
                const float z = (p.water - (b.t.f(i).y - nr.z)) / (2.0f * nr.z);
                if (z >= 0.0f && z <= 1.0f) {
                    dfy = -kWaterBuoyancy * nr.x * p.gravity * dp.y / (2.0f * nr.z);
                }
            }
            float2 dv = d.vel(i);
            dv.x += C::h * dfp.x * im;
            dv.y += C::h * (dfp.y + dfy) * im;
            if (du_mass) {
                // The world forces are a mass times an acceleration, so only
                // the muscle force (the kept A.force entry) feels the mass.
                const float2 F = reinterpret_cast<const float2*>(&L.base[(bw.A.force + i / 2u) * 32u])[i % 2u];
                const float dim = dinv(i, im);
                dv.x += C::h * F.x * dim;
                dv.y += C::h * F.y * dim;
            }
            if (b.w.has(CE_FLAG_AIR)) {
                dv.x *= b.p.air_sub;
                dv.y *= b.p.air_sub;
            }
            d.f(i) = dp;
            d.vel(i) = dv;
            d.pos(i) = make_float2(dp.x + C::h * dv.x, dp.y + C::h * dv.y);
        }
    }

    // Tangent of the bone lengths (Creature::bone_item), bone by bone from
    // the positions each bone saw (A.bones).
    __device__ __forceinline__ void bones_tan() const {
        const Body& b = bw.b;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const unsigned bones = b.r.nodes - 1u;
        for (unsigned j = 0u; j < bones; j++) {
            const float4 ba = L.get(S.bone + 2u * j);
            const float4 pre = L.get(bw.A.bones + j);
            const unsigned i0 = __float_as_uint(ba.x), i1 = j + 1u;
            const float dx = pre.z - pre.x, dy = pre.w - pre.y;
            const float len0 = sqrtf(dx * dx + dy * dy);
            const float len = fmaxf(len0, 1e-9f);
            const float w0 = ba.z, w1 = ba.w;
            const float sc = (len - ba.y) / ((w0 + w1) * len);
            const float2 l0 = d.pos(i0), l1 = d.pos(i1);
            const float ddx = l1.x - l0.x, ddy = l1.y - l0.y;
            const float dlen = len0 >= 1e-9f ? (dx * ddx + dy * ddy) / len : 0.0f;
            const float dw0 = du_mass ? dinv(i0, w0) : 0.0f, dw1 = du_mass ? dinv(i1, w1) : 0.0f;
            const float ds = dlen * ba.y / ((w0 + w1) * len * len) - sc * (dw0 + dw1) / (w0 + w1);
            const float mx = ds * dx + sc * ddx, my = ds * dy + sc * ddy;
            d.pos(i0) = make_float2(l0.x + w0 * mx + dw0 * sc * dx, l0.y + w0 * my + dw0 * sc * dy);
            d.pos(i1) = make_float2(l1.x - w1 * mx - dw1 * sc * dx, l1.y - w1 * my - dw1 * sc * dy);
        }
    }

    // d g of a joint gradient vector g = perp(w) / |w|^2 (Backward::perp_back
    // transposed).
    __device__ __forceinline__ static float2 perp_tan(float2 w, float ww, float2 gw, float2 dw) {
        float2 dg = make_float2(-dw.y / ww, dw.x / ww);
        if (ww >= 1e-12f && w.x * w.x + w.y * w.y >= 1e-12f) {
            const float c = 2.0f * (w.x * dw.x + w.y * dw.y) / ww;
            dg.x -= c * gw.x;
            dg.y -= c * gw.y;
        }
        return dg;
    }

    // Tangents of a joint's gradient vectors (tip, far, hub) from the
    // positions u = parent tip - parent pivot, v = tip - hub and their
    // tangents; gv are the vectors themselves (Body::joint).
    __device__ __forceinline__ static void geometry_tan(float2 u, float2 v, float2 du, float2 dv, bool at_head,
                                                        float2 (&gv)[3], float2 (&dg)[3]) {
        const float uu = fmaxf(u.x * u.x + u.y * u.y, 1e-12f), vv = fmaxf(v.x * v.x + v.y * v.y, 1e-12f);
        const float2 g_u = make_float2(-u.y / uu, u.x / uu);
        gv[0] = make_float2(-v.y / vv, v.x / vv);
        gv[1] = at_head ? make_float2(-g_u.x, -g_u.y) : g_u;
        gv[2] = make_float2(-(gv[0].x + gv[1].x), -(gv[0].y + gv[1].y));
        dg[0] = perp_tan(v, vv, gv[0], dv);
        const float2 dgu = perp_tan(u, uu, g_u, du);
        dg[1] = at_head ? make_float2(-dgu.x, -dgu.y) : dgu;
        dg[2] = make_float2(-(dg[0].x + dg[1].x), -(dg[0].y + dg[1].y));
    }

    // Adds w_n (dlam g_n + lam dg_n) + dw_n lam g_n to the tangents of the
    // three nodes (w_n their inverse masses).
    template <bool VEL>
    __device__ __forceinline__ void push_tan(const unsigned (&node)[3], const float (&wn)[3], const float (&dwn)[3],
                                             const float2 (&gv)[3], const float2 (&dg)[3], float lam, float dlam) const {
        for (int n = 0; n < 3; n++) {
            float2& e = VEL ? d.vel(node[n]) : d.pos(node[n]);
            const float2 o = e;
            e = make_float2(o.x + wn[n] * (dlam * gv[n].x + lam * dg[n].x) + dwn[n] * lam * gv[n].x,
                            o.y + wn[n] * (dlam * gv[n].y + lam * dg[n].y) + dwn[n] * lam * gv[n].y);
        }
    }

    // Tangent of the joint limits (Creature::limit_item) on the joints that
    // were pushed, in the pass's order, from the positions each joint's test
    // saw (A.joints).
    __device__ __forceinline__ void joints_tan(unsigned violated) const {
        const Body& b = bw.b;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const unsigned bones = b.r.nodes - 1u;
        for (unsigned j = 1u; j < bones; j++) {
            if (((violated >> j) & 1u) == 0u) {
                continue;
            }
            const float4 ra = L.get(S.joint + 2u * j), rb = L.get(S.joint + 2u * j + 1u);
            const float4 e0 = L.get(bw.A.joints + 2u * j), e1 = L.get(bw.A.joints + 2u * j + 1u);
            const unsigned topo = __float_as_uint(ra.x);
            const unsigned hub = topo & 31u, ptip = (topo >> 5u) & 31u, ppivot = (topo >> 10u) & 31u;
            const unsigned far = (topo >> 15u) & 31u, tip = j + 1u;
            const bool at_head = ((topo >> 20u) & 1u) != 0u;
            const float2 u = make_float2(e0.x - e0.z, e0.y - e0.w), v = make_float2(e1.x - e1.z, e1.y - e1.w);
            const float2 dpt = d.pos(ptip), dpp = d.pos(ppivot), dct = d.pos(tip), dch = d.pos(hub);
            const float2 du = make_float2(dpt.x - dpp.x, dpt.y - dpp.y), dv = make_float2(dct.x - dch.x, dct.y - dch.y);
            const float turn = atan2f(u.x * v.y - u.y * v.x, u.x * v.x + u.y * v.y);
            const float mid = ra.w;
            const float angle = mid + wrapf(turn - mid);
            float error = 0.0f;
            if (angle < ra.y) {
                error = angle - ra.y;
            }
            if (angle > ra.z) {
                error = angle - ra.z;
            }
            const float cr = u.x * v.y - u.y * v.x, dt = u.x * v.x + u.y * v.y;
            const float den = cr * cr + dt * dt;
            float derror = 0.0f;
            if (den > 0.0f) {
                const float dcr = du.x * v.y + u.x * dv.y - du.y * v.x - u.y * dv.x;
                const float ddt = du.x * v.x + du.y * v.y + u.x * dv.x + u.y * dv.y;
                derror = (dt * dcr - cr * ddt) / den;
            }
            float2 gv[3], dg[3];
            geometry_tan(u, v, du, dv, at_head, gv, dg);
            const float wn[3] = {rb.x, rb.y, rb.z};
            const unsigned node[3] = {tip, far, hub};
            float dwn[3] = {0.0f, 0.0f, 0.0f};
            float wgt = 0.0f, dwgt = 0.0f;
            for (int n = 0; n < 3; n++) {
                if (du_mass) {
                    dwn[n] = dinv(node[n], wn[n]);
                }
                const float gg = gv[n].x * gv[n].x + gv[n].y * gv[n].y;
                wgt += wn[n] * gg;
                dwgt += 2.0f * wn[n] * (gv[n].x * dg[n].x + gv[n].y * dg[n].y) + dwn[n] * gg;
            }
            const float lam = -error / wgt;
            const float dlam = -derror / wgt + error * dwgt / (wgt * wgt);
            push_tan<false>(node, wn, dwn, gv, dg, lam, dlam);
        }
    }

    // Tangent of the ground contact (Creature::solve_ground) of the nodes
    // that touched, from the positions before it (A.pj) and the substep's
    // start positions (the forward force table), then of the velocities
    // v = (q - q0) / h.
    __device__ __forceinline__ void ground_tan(unsigned touch, unsigned slip) const {
        const Body& b = bw.b;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const ce_params& p = b.p;
        for (unsigned i = 0u; i < b.r.nodes; i++) {
            if (((touch >> i) & 1u) == 0u) {
                continue;
            }
            const float4 nr = L.get(S.node + i);
            const float* pj = reinterpret_cast<const float*>(&L.base[(bw.A.pj + i / 2u) * 32u]) + 2u * (i % 2u);
            const float2 q = make_float2(pj[0], pj[1]), f0 = b.t.f(i);
            const typename B::Contact c = bw.contact(q, f0, nr);
            const float Sl = c.gr.y, sec = c.secant;
            const float2 dq = d.pos(i), df0 = d.f(i);
            const float dh = Sl * dq.x;
            const float dS = ground_curvature(b.w, q.x, b.r.amp, b.r.qphase) * dq.x;
            const float dsec = Sl * dS / sec;
            const float dnx = -dS / sec + Sl * dsec / (sec * sec), dny = -dsec / (sec * sec);
            const float ddepth = -((dq.y - dh) / sec - (q.y - c.gr.x) * dsec / (sec * sec));
            float dmu = du_friction ? du_friction[i] * p.friction * c.ice : 0.0f;
            if (b.w.has(CE_FLAG_ICE)) {
                dmu -= nr.w * p.friction * p.patches * ice_slope(q.x) * dq.x;
            }
            const float2 dq1 = make_float2(dq.x + dnx * c.depth + c.n.x * ddepth, dq.y + dny * c.depth + c.n.y * ddepth);
            const float tx = c.n.y, ty = -c.n.x, dtx = dny, dty = -dnx;
            const float dslide = (dq1.x - df0.x) * tx + (dq1.y - df0.y) * ty + (c.q1.x - f0.x) * dtx +
                                 (c.q1.y - f0.y) * dty;
            const bool slipped = ((slip >> i) & 1u) != 0u;
            const float budget = c.mu * c.depth;
            const float back = slipped ? copysignf(budget, c.slide) : c.slide;
            const float dback = slipped ? (c.slide < 0.0f ? -1.0f : 1.0f) * (dmu * c.depth + c.mu * ddepth) : dslide;
            d.pos(i) = make_float2(dq1.x - dtx * back - tx * dback, dq1.y - dty * back - ty * dback);
        }
        for (unsigned i = 0u; i < b.r.nodes; i++) {
            const float2 dq = d.pos(i), df0 = d.f(i);
            d.vel(i) = make_float2((dq.x - df0.x) * C::inv_h, (dq.y - df0.y) * C::inv_h);
        }
    }

    // Tangent of the joint damping (Creature::damp_item), joint by joint
    // from the velocities each joint saw (A.damp), on the substep's final
    // positions (in the tables).
    __device__ __forceinline__ void damp_tan() const {
        const Body& b = bw.b;
        const Lines& L = b.L;
        const SlotLayout& S = b.S;
        const NodeTables& t = b.t;
        const unsigned bones = b.r.nodes - 1u;
        const float share = fminf(C::h * kInvJointDamping, 1.0f);
        for (unsigned j = 1u; j < bones; j++) {
            const float4 ra = L.get(S.joint + 2u * j), rb = L.get(S.joint + 2u * j + 1u);
            if (__float_as_uint(ra.x) == kNone) {
                continue;
            }
            const typename Body::Joint k = b.joint(j, ra, rb, false);
            const float wgt = Body::joint_weight(k);
            if (!(wgt > 0.0f)) {
                continue;
            }
            const unsigned topo = __float_as_uint(ra.x);
            const unsigned ptip = (topo >> 5u) & 31u, ppivot = (topo >> 10u) & 31u;
            const bool at_head = ((topo >> 20u) & 1u) != 0u;
            const float4 d0 = L.get(bw.A.damp + 2u * j), d1 = L.get(bw.A.damp + 2u * j + 1u);
            const float2 vn[3] = {make_float2(d0.x, d0.y), make_float2(d0.z, d0.w), make_float2(d1.x, d1.y)};
            const float2 pt = t.pos(ptip), pp = t.pos(ppivot), ct = t.pos(k.tip), ch = t.pos(k.hub);
            const float2 dpt = d.pos(ptip), dpp = d.pos(ppivot), dct = d.pos(k.tip), dch = d.pos(k.hub);
            float2 gv[3], dg[3];
            geometry_tan(make_float2(pt.x - pp.x, pt.y - pp.y), make_float2(ct.x - ch.x, ct.y - ch.y),
                         make_float2(dpt.x - dpp.x, dpt.y - dpp.y), make_float2(dct.x - dch.x, dct.y - dch.y), at_head,
                         gv, dg);
            const unsigned node[3] = {k.tip, k.far, k.hub};
            const float wn[3] = {k.w_tip, k.w_far, k.w_hub};
            float dwn[3] = {0.0f, 0.0f, 0.0f};
            float rate = 0.0f, drate = 0.0f, dwgt = 0.0f;
            for (int n = 0; n < 3; n++) {
                if (du_mass) {
                    dwn[n] = dinv(node[n], wn[n]);
                }
                const float2 dvn = d.vel(node[n]);
                rate += gv[n].x * vn[n].x + gv[n].y * vn[n].y;
                drate += dg[n].x * vn[n].x + dg[n].y * vn[n].y + gv[n].x * dvn.x + gv[n].y * dvn.y;
                dwgt += 2.0f * wn[n] * (gv[n].x * dg[n].x + gv[n].y * dg[n].y) +
                        dwn[n] * (gv[n].x * gv[n].x + gv[n].y * gv[n].y);
            }
            const float lam = -share * rate / wgt;
            const float dlam = -share * drate / wgt + share * rate * dwgt / (wgt * wgt);
            push_tan<true>(node, wn, dwn, gv, dg, lam, dlam);
        }
    }

    // Runs creature `cidx`'s trial with the tangent of its start positions
    // `dstart` (2 x rows floats, (x, y) per node row, null for 0) and of the
    // parameters (du_muscle, du_friction) and returns d fitness; 0 for a
    // trial that failed or ran no step.
    __device__ __forceinline__ float run(unsigned cidx, const float* dstart) const {
        const Body& b = bw.b;
        const KernelArgs& a = bw.a;
        LaneRegs& r = b.r;
        B::T::begin(b, a, cidx, 0u);
        const unsigned end = a.ends[cidx];
        if (end == 0u || !(a.results[cidx].fitness > -1e19f)) {
            return 0.0f;
        }
        for (unsigned i = 0u; i < r.nodes; i++) {
            d.pos(i) = dstart ? make_float2(dstart[2u * i], dstart[2u * i + 1u]) : make_float2(0.0f, 0.0f);
            d.vel(i) = make_float2(0.0f, 0.0f);
        }
        for (unsigned k = 0u; k < r.muscles; k++) {
            d.muscle(k) = make_float2(0.0f, 0.0f);
        }
        for (unsigned s = 0u; s < end; s++) {
            b.muscle_demands((float)s * C::dt);
            demands_tan((float)s * C::dt);
            for (unsigned q = 0u; q < 16u; q++) {
                muscles_tan();
                unsigned touch, slip;
                const unsigned violated = bw.substep_kept(touch, slip);
                drag_tan();
                integrate_tan();
                bones_tan();
                joints_tan(violated);
                ground_tan(touch, slip);
                damp_tan();
            }
        }
        // Fitness com_x = sum m x / sum m.
        float dfit = 0.0f, com_x = 0.0f;
        for (unsigned i = 0u; i < r.nodes; i++) {
            const float m = b.L.get(b.S.node + i).x;
            dfit += m * d.pos(i).x;
            com_x += m * b.t.pos(i).x;
        }
        com_x *= r.inv_mass;
        if (du_mass) {
            for (unsigned i = 0u; i < r.nodes; i++) {
                dfit += dmass(i) * (b.t.pos(i).x - com_x);
            }
        }
        return dfit * r.inv_mass;
    }
};

template <class W, int RATE>
__global__ void __launch_bounds__(kBlock, 1) tangent_kernel(const KernelArgs a, const ce_params p, const float* dstart,
                                                            const float* dmuscle, const float* dfriction,
                                                            const float* dmass, float* dfitness) {
    extern __shared__ float4 smem[];
    using B = Backward<W, RATE>;
    const unsigned threads = blockDim.x;
    float2* const tables = reinterpret_cast<float2*>(smem) + threadIdx.x;
    // Tables of rows x threads entries: positions, velocities, forces (the
    // forward run's), then their tangents; then the muscles' (energy,
    // demand) and their tangents.
    const size_t node_table = (size_t)a.rows * threads, muscle_table = (size_t)(a.mm > 0u ? a.mm : 1u) * threads;
    float2* const muscles = reinterpret_cast<float2*>(smem) + 6u * node_table + threadIdx.x;
    const NodeTables tab{tables, tables + node_table, tables + 2u * node_table, muscles};
    const NodeTables tan{tables + 3u * node_table, tables + 4u * node_table, tables + 5u * node_table,
                         muscles + muscle_table};
    const SlotLayout S = SlotLayout::make(a.rows, a.mm, false);
    const AdjointLayout A = AdjointLayout::make(a.rows, a.mm);
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = (blockIdx.x * threads + threadIdx.x) >> 5u;
    const unsigned warps_total = gridDim.x * (threads >> 5u);
    const Lines L = Lines::make(a.scratch + (size_t)warp * A.lines * 32u, lane);
    const Tape tape{nullptr, 0u};
    const AdjointArgs x{nullptr, nullptr, nullptr, nullptr};
    const W w{};
    LaneRegs r;
    const typename B::Body body{w, p, tab, L, S, r};
    unsigned end = 0u, seg = 0u;
    float weight = 1.0f;
    const B back{body, tan, nullptr, A, tape, a, x, end, seg, weight};
    const size_t per = 2u * (size_t)a.rows;
    Claim claim(a, lane, warp, warps_total);
    for (;;) {
        const unsigned mine = claim.next(false);
        if (__ballot_sync(kFull, mine != kNone) == 0u) {
            if (claim.drained) {
                break;
            }
            continue;
        }
        if (mine != kNone) {
            const unsigned cidx = a.order ? __ldg(a.order + mine) : p.base + mine;
            const Tangent<W, RATE> tl{back, tan, dmuscle ? dmuscle + (size_t)cidx * kGradMuscle * a.mm : nullptr,
                                      dfriction ? dfriction + (size_t)cidx * a.rows : nullptr,
                                      dmass ? dmass + (size_t)cidx * a.rows : nullptr};
            dfitness[cidx] = tl.run(cidx, dstart ? dstart + (size_t)cidx * per : nullptr);
        }
    }
}
