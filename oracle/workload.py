"""The bench's seeded synthetic workloads, restated without the engine.

TEST INFRASTRUCTURE ONLY (tests/, bench.py's CPU arms): the CPU baseline and
the reference arm build their inputs here so that their processes never load
the engine's library.  This is a line-by-line restatement of the engine's
host trace generator (SplitMix64, Steele, Lea & Flood 2014, with Box-Muller
normals in double precision, and the models' ground-truth dynamics): the same
seeds give the same parameters, controls, measurements and ground truth.
Python's math functions are the C library's, evaluated in the same order, so
the values agree with the engine's generator (tests/test_oracle_workload.py).
"""
import math
from types import SimpleNamespace

import numpy as np

MASK = (1 << 64) - 1
MODEL_UNICYCLE, MODEL_DHARM, MODEL_BEACON = 0, 1, 3
NUM_STATE = {MODEL_UNICYCLE: 3, MODEL_DHARM: 12, MODEL_BEACON: 3}


class SplitMix64:
    def __init__(self, s):
        self.s = s & MASK

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def unif(self):
        return float(self.next() >> 11) * (1.0 / 9007199254740992.0)

    def gauss(self):
        u1 = 1.0 - self.unif()
        u2 = self.unif()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def _f32(x):
    return float(np.float32(x))


def _wrap(a):
    return a - 2.0 * math.pi * math.floor((a + math.pi) / (2.0 * math.pi))


def unicycle_params(seed, num_landmarks=4):
    """Range/bearing unicycle: dt 0.1, process noise (0.05, 0.05, 0.01), sigma_r
    0.2, sigma_b 0.05, landmarks uniform in [-10, 10]^2 from the seed."""
    r = SplitMix64(0x4C414E444D41524B ^ (seed << 20))
    lm = [[0.0, 0.0] for _ in range(8)]
    for j in range(num_landmarks):
        lm[j][0] = _f32(-10.0 + 20.0 * r.unif())
        lm[j][1] = _f32(-10.0 + 20.0 * r.unif())
    return SimpleNamespace(dt=_f32(0.1), sigma_q=[_f32(0.05), _f32(0.05), _f32(0.01)], sigma_range=_f32(0.2),
                           sigma_bearing=_f32(0.05), num_landmarks=num_landmarks, landmarks=lm,
                           init_state=[0.0, 0.0, 0.0])


def dharm_params(seed):
    """6-joint DH arm: dt 0.01, velocity noise 0.01, position sigma 5 mm, angle
    sigma 0.02; a uniform [0.2, 0.6], twists from {0, +-pi/2}, from the seed."""
    r = SplitMix64(0x4448415241524D53 ^ (seed << 20))
    alphas = (0.0, math.pi / 2, -math.pi / 2)
    a, alpha = [0.0] * 6, [0.0] * 6
    for i in range(6):
        a[i] = _f32(0.2 + 0.4 * r.unif())
        k = int(3.0 * r.unif())
        alpha[i] = _f32(alphas[min(k, 2)])
    init = [0.0] * 12
    for i in range(6):
        init[i] = _f32(-math.pi / 2 + math.pi * r.unif())
        init[6 + i] = _f32(-0.5 + r.unif())
    return SimpleNamespace(dt=_f32(0.01), sigma_qd=_f32(0.01), sigma_pos=_f32(0.005), sigma_ang=_f32(0.02),
                           a=a, alpha=alpha, d=[0.0] * 6, init_state=init)


def beacon_params():
    """The reference unicycle program's ten beacons, noise and start pose."""
    bx = [12, 12, 13, 14, 16, 16, 18, 20, 20, 20]
    by = [12, 37, 25, 18, 12, 37, 30, 12, 25, 37]
    bc = [[0.0, 0.0, 0.0] for _ in range(16)]
    for j in range(10):
        bc[j] = [float(bx[j]), float(by[j]), 3.0]
    return SimpleNamespace(dt=1.0, noise=[_f32(0.5), _f32(0.1), _f32(0.01)], sigma_range=_f32(math.sqrt(0.5)),
                           num_beacons=10, beacons=bc, init_state=[20.0, 40.0, _f32(-math.pi / 2)])


def params(model, seed):
    if model == MODEL_UNICYCLE:
        return unicycle_params(seed)
    if model == MODEL_DHARM:
        return dharm_params(seed)
    return beacon_params()


def _dh_fk(P, q):
    R = [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]
    p = [0.0, 0.0, 0.0]
    for i in range(6):
        ct, st = math.cos(q[i]), math.sin(q[i])
        ca, sa = math.cos(P.alpha[i]), math.sin(P.alpha[i])
        Ra = [[ct, -st * ca, st * sa], [st, ct * ca, -ct * sa], [0.0, sa, ca]]
        pa = [P.a[i] * ct, P.a[i] * st, P.d[i]]
        Rn = [[R[r][0] * Ra[0][k] + R[r][1] * Ra[1][k] + R[r][2] * Ra[2][k] for k in range(3)] for r in range(3)]
        pn = [R[r][0] * pa[0] + R[r][1] * pa[1] + R[r][2] * pa[2] + p[r] for r in range(3)]
        R, p = Rn, pn
    return [p[0], p[1], p[2], math.atan2(R[1][0], R[0][0]),
            math.atan2(-R[2][0], math.sqrt(R[2][1] * R[2][1] + R[2][2] * R[2][2])), math.atan2(R[2][1], R[2][2])]


def make_trace(model, P, seed, steps):
    """(control [steps, 8], meas [steps, 16], dt [steps], truth [steps, S]) as float32."""
    r = SplitMix64(0x5452414345534544 ^ (seed << 24) ^ model)
    S = NUM_STATE[model]
    control = np.zeros((steps, 8), np.float32)
    meas = np.zeros((steps, 16), np.float32)
    dtv = np.zeros(steps, np.float32)
    truth = np.zeros((steps, S), np.float32)
    if model == MODEL_UNICYCLE:
        L = P.num_landmarks
        x, y, th = (float(v) for v in P.init_state[:3])
        dt = float(P.dt)
        for k in range(steps):
            t = k * dt
            v, w = 1.0, 0.3 * math.sin(0.05 * t)
            wd = w * dt
            if abs(wd) < 1e-4:
                A = v * dt * (1.0 - wd * wd / 6.0)
                B = v * dt * (wd / 2.0)
            else:
                A = v * math.sin(wd) / w
                B = v * (1.0 - math.cos(wd)) / w
            c, s = math.cos(th), math.sin(th)
            x = x + A * c - B * s + P.sigma_q[0] * r.gauss()
            y = y + A * s + B * c + P.sigma_q[1] * r.gauss()
            th = _wrap(th + wd + P.sigma_q[2] * r.gauss())
            dtv[k], control[k, 0], control[k, 1] = dt, v, w
            for j in range(L):
                dx, dy = P.landmarks[j][0] - x, P.landmarks[j][1] - y
                meas[k, j] = math.sqrt(dx * dx + dy * dy) + P.sigma_range * r.gauss()
                meas[k, L + j] = _wrap(math.atan2(dy, dx) - th + P.sigma_bearing * r.gauss())
            truth[k] = (x, y, th)
    elif model == MODEL_DHARM:
        q = [float(v) for v in P.init_state[:6]]
        qd = [float(v) for v in P.init_state[6:12]]
        for k in range(steps):
            for i in range(6):
                q[i] = _wrap(q[i] + qd[i] * P.dt)
                qd[i] = qd[i] + P.sigma_qd * r.gauss()
            z = _dh_fk(P, q)
            dtv[k] = P.dt
            for i in range(3):
                meas[k, i] = z[i] + P.sigma_pos * r.gauss()
            for i in range(3, 6):
                meas[k, i] = _wrap(z[i] + P.sigma_ang * r.gauss())
            truth[k, :6] = q
            truth[k, 6:] = qd
    elif model == MODEL_BEACON:
        L = P.num_beacons
        x, y, th = (float(v) for v in P.init_state[:3])
        dt = float(P.dt)
        for k in range(steps):
            v = abs(0.3 + 0.1 * r.gauss())
            w = 0.3 * r.gauss()
            h = 0.5 * w * dt
            sc = 1.0 if abs(h) < 1e-8 else math.sin(h) / h
            x += v * dt * sc * math.cos(th + h)
            y += v * dt * sc * math.sin(th + h)
            th = _wrap(th + w * dt)
            dtv[k], control[k, 0], control[k, 1] = dt, v, w
            for j in range(L):
                dx, dy, dz = x - P.beacons[j][0], y - P.beacons[j][1], P.beacons[j][2]
                meas[k, j] = math.sqrt(dx * dx + dy * dy + dz * dz) + P.sigma_range * r.gauss()
            truth[k] = (x, y, th)
    else:
        raise ValueError("no generator for model %d" % model)
    return control, meas, dtv, truth
