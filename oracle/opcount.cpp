// TEST AND MEASUREMENT INFRASTRUCTURE ONLY: counts the algorithmic
// floating-point operations of one march step of the reference algorithm
// (Geodesic.h:42-59 rayDerivative/rayStep, :89-91 rayPosition, :177-181
// rayStepLength, march.metal:67-80 path length; Kerr.h:63-99, 150-154,
// 177-186; march.metal:81-102 gather) by running it once on a scalar type
// that counts every add, subtract, multiply, divide, square root and
// transcendental as one operation (a fused multiply-add written as such
// would count two; the reference writes none). Comparisons, min, max and
// abs are not counted. The counts are the per-ray-step FLOP figures the
// bench divides by the FP32 peak for its roofline.
//
// Build: g++ -O1 -std=c++17 opcount.cpp -o opcount ; prints JSON.
#include <cmath>
#include <cstdio>

static long g_ops = 0;

struct N {
    double v;
    N(double x = 0) : v(x) {}
};
static N operator+(N a, N b) { ++g_ops; return N(a.v + b.v); }
static N operator-(N a, N b) { ++g_ops; return N(a.v - b.v); }
static N operator*(N a, N b) { ++g_ops; return N(a.v * b.v); }
static N operator/(N a, N b) { ++g_ops; return N(a.v / b.v); }
static N operator-(N a) { return N(-a.v); }
static bool operator<(N a, N b) { return a.v < b.v; }
static bool operator>(N a, N b) { return a.v > b.v; }
static N Sqrt(N a) { ++g_ops; return N(std::sqrt(a.v)); }
static N Sin(N a) { ++g_ops; return N(std::sin(a.v)); }
static N Cos(N a) { ++g_ops; return N(std::cos(a.v)); }
static N Exp(N a) { ++g_ops; return N(std::exp(a.v)); }
static N Tanh(N a) { ++g_ops; return N(std::tanh(a.v)); }
static N Abs(N a) { return N(std::fabs(a.v)); }
static N Max(N a, N b) { return a.v > b.v ? a : b; }
static N Min(N a, N b) { return a.v < b.v ? a : b; }

struct S { N v, r, phi, vd, rd, pd; };
static S add(S a, S b) { return {a.v + b.v, a.r + b.r, a.phi + b.phi, a.vd + b.vd, a.rd + b.rd, a.pd + b.pd}; }
static S scale(S a, N s) { return {a.v * s, a.r * s, a.phi * s, a.vd * s, a.rd * s, a.pd * s}; }
static N f(N r) { return N(1.0) - N(2.0) / r; }

// Geodesic.h:42-49
static S deriv(S s) {
    N r = s.r;
    N r2 = r * r;
    N vdd = -s.vd * s.vd / r2 + r * s.pd * s.pd;
    N rdd = N(2.0) * s.rd * s.vd / r2 + f(r) * (r * s.pd * s.pd - s.vd * s.vd / r2);
    N pdd = N(-2.0) * s.rd * s.pd / r;
    return {s.vd, s.rd, s.pd, vdd, rdd, pdd};
}

// Geodesic.h:52-59
static S rk4(S s, N h) {
    S k1 = deriv(s);
    S k2 = deriv(add(s, scale(k1, N(0.5) * h)));
    S k3 = deriv(add(s, scale(k2, N(0.5) * h)));
    S k4 = deriv(add(s, scale(k3, h)));
    S sum = add(add(k1, scale(k2, N(2.0))), add(scale(k3, N(2.0)), k4));
    return add(s, scale(sum, h / N(6.0)));
}

struct V { N x, y, z; };
static V vadd(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static V vsub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static V vmul(V a, N s) { return {a.x * s, a.y * s, a.z * s}; }
static N vdot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static N vlen(V a) { return Sqrt(vdot(a, a)); }

int main() {
    long step = 0, position = 0, policy = 0, path = 0, gather = 0, direction = 0, kerr_step = 0, kerr_extra = 0;
    S s{0, 20, 0.3, 1.1, -0.8, 0.01};
    V e1{1, 0, 0}, e2{0, 1, 0}, prev{19, 1, 0.5};
    N h(0.4);
    g_ops = 0; s = rk4(s, h); step = g_ops;
    // rayPosition (Geodesic.h:89-91)
    g_ops = 0; V pos = vmul(vadd(vmul(e1, Cos(s.phi)), vmul(e2, Sin(s.phi))), s.r); position = g_ops;
    // rayStepLength (Geodesic.h:177-181): one clamp product each branch
    g_ops = 0; { N coarse = Min(Max(N(0.1) * s.r, N(0.02)), N(3.0)); N z = Abs(pos.z);
                 if (z > N(6.0) + coarse) {} N fine = Min(Max(N(0.02) * s.r, N(0.02)), N(0.5)); (void)fine; } policy = g_ops;
    // path length and travelled (march.metal:78-79)
    g_ops = 0; { N pl = vlen(vsub(pos, prev)); N travelled = N(0) + pl; (void)travelled; } path = g_ops;
    // rayDirection (Geodesic.h:94-100)
    g_ops = 0; { N c = Cos(s.phi), sn = Sin(s.phi); V radial = vadd(vmul(e1, c), vmul(e2, sn));
                 V tang = vadd(vmul(e1, -sn), vmul(e2, c));
                 V local = vadd(vmul(radial, s.rd / Sqrt(Max(f(s.r), N(1e-6)))), vmul(tang, s.r * s.pd));
                 N len = vlen(local); V d = vmul(local, N(1.0) / len); (void)d; } direction = g_ops;
    // gather of one in-slab sample (march.metal:81-102) incl. sampleVolume's
    // coordinate transform and redshiftFactor (Geodesic.h:225-236), without
    // the direction above
    g_ops = 0; {
        N half(30); V uvw = vmul(vadd(pos, V{half, half, half}), N(1.0) / (N(2.0) * half)); (void)uvw;
        V gas{0.1, 0.2, 0.0}; N density(50), path_len(0.3), T(0.9), travelled(40);
        V dir{0.3, 0.4, 0.5}; V em{0.1, 0.2, 0.3};
        N fr = f(s.r);
        N mag = vlen(gas); N speed = Min(mag, N(8.0));
        N beta = N(0.85) * Tanh(speed / N(0.85));
        V vel = vmul(gas, beta / mag);
        N gamma = N(1.0) / Sqrt(N(1.0) - beta * beta);
        N g = Sqrt(Max(fr, N(0))) / (gamma * (N(1.0) + vdot(dir, vel)));
        N gravity = Sqrt(Max(fr, N(0)));
        N bulk = Min(density / N(40.0), N(1.0));
        N gr3 = gravity * gravity * gravity;
        N g3 = gr3 + (g * g * g - gr3) * bulk;
        N alpha = N(1.0) - Exp(-N(5e-4) * density * path_len);
        V contrib = vmul(em, T * g3 * path_len);
        V color = vadd(V{0, 0, 0}, contrib);
        N w = contrib.x * N(0.2126) + contrib.y * N(0.7152) + contrib.z * N(0.0722);
        N wd = N(0) + w * travelled; N dw = N(0) + w; T = T * (N(1.0) - alpha);
        (void)color; (void)wd; (void)dw;
    } gather = g_ops;
    // Kerr: kerrStep (Kerr.h:63-99) with sin/cos per derivative
    {
        N a(0.9);
        struct K { N r, th, ph, pr, pt; };
        N E(1.0), L(3.0);
        auto kd = [&](K s) {
            N r = s.r;
            N delta = r * r - N(2.0) * r + a * a;
            N ct = Cos(s.th), st = Sin(s.th);
            N sigma = r * r + a * a * ct * ct;
            N dprime = N(2.0) * r - N(2.0);
            N sin2 = Max(st * st, N(1e-8));
            N p = (r * r + a * a) * E - a * L;
            N g = L * L / sin2 - N(2.0) * a * E * L + a * a * E * E * sin2;
            N F = delta * s.pr * s.pr + s.pt * s.pt - p * p / delta + g;
            N ham = F / (N(2.0) * sigma);
            N pp = N(2.0) * r * E;
            N fr = dprime * s.pr * s.pr - N(2.0) * p * pp / delta + p * p * dprime / (delta * delta);
            N fth = N(-2.0) * L * L * ct / (sin2 * Max(st, N(1e-4))) + N(2.0) * a * a * E * E * st * ct;
            N sr = N(2.0) * r, sth = N(-2.0) * a * a * st * ct;
            K o;
            o.r = delta * s.pr / sigma;
            o.th = s.pt / sigma;
            o.ph = (a * p / delta + L / sin2 - a * E) / sigma;
            o.pr = -(fr / (N(2.0) * sigma) - ham * sr / sigma);
            o.pt = -(fth / (N(2.0) * sigma) - ham * sth / sigma);
            return o;
        };
        auto kadd = [](K x, K y) { return K{x.r + y.r, x.th + y.th, x.ph + y.ph, x.pr + y.pr, x.pt + y.pt}; };
        auto kscale = [](K x, N f) { return K{x.r * f, x.th * f, x.ph * f, x.pr * f, x.pt * f}; };
        K ks{20, 1.2, 0.3, -0.9, 0.2};
        g_ops = 0;
        K k1 = kd(ks);
        K k2 = kd(kadd(ks, kscale(k1, N(0.5) * h)));
        K k3 = kd(kadd(ks, kscale(k2, N(0.5) * h)));
        K k4 = kd(kadd(ks, kscale(k3, h)));
        K sum = kadd(kadd(k1, kscale(k2, N(2.0))), kadd(kscale(k3, N(2.0)), k4));
        ks = kadd(ks, kscale(sum, h / N(6.0)));
        kerr_step = g_ops;
        // per-step extras (march.metal:142-149): step length, position, path,
        // Carter and null-residual gauges
        g_ops = 0;
        {
            N above = ks.r - (N(1.0) + Sqrt(Max(N(1.0) - a * a, N(0))));
            N nearv = N(0.2) * above;
            N pole = Min(Max(Sin(ks.th) / N(0.08), N(0.05)), N(1.0));
            N hh = Min(Max(Min(N(0.02) * ks.r, nearv) * pole, N(0.002)), N(0.5)); (void)hh;
            N radial = Sqrt(ks.r * ks.r + a * a); N st = Sin(ks.th), ct = Cos(ks.th);
            V p3{radial * st * Cos(ks.ph), radial * st * Sin(ks.ph), ks.r * ct};
            N pl = vlen(vsub(p3, prev)); N trav = N(0) + pl; (void)trav;
            N sin2 = Max(st * st, N(1e-8));
            N term = L * L / sin2 - a * a * E * E;
            N Q = ks.pt * ks.pt + ct * ct * term;
            N Q0(10), scl(10);
            N cd = Abs(Q - Q0) / scl;
            N delta = ks.r * ks.r - N(2.0) * ks.r + a * a;
            N p = (ks.r * ks.r + a * a) * E - a * L;
            N g = L * L / sin2 - N(2.0) * a * E * L + a * a * E * E * sin2;
            N res = delta * ks.pr * ks.pr + ks.pt * ks.pt - p * p / delta + g;
            N nd = Abs(res) / (scl * Max(ks.r * ks.r, N(1.0)));
            (void)cd; (void)nd;
        }
        kerr_extra = g_ops;
    }
    std::printf("{\"schwarzschild_rk4\": %ld, \"position\": %ld, \"step_policy\": %ld, \"path\": %ld, "
                "\"schwarzschild_step\": %ld, \"direction\": %ld, \"gather\": %ld, \"kerr_rk4\": %ld, "
                "\"kerr_extra\": %ld, \"kerr_step\": %ld}\n",
                step, position, policy, path, step + position + policy + path, direction, gather, kerr_step, kerr_extra,
                kerr_step + kerr_extra);
    return 0;
}
