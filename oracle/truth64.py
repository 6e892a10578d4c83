"""Float64 truth for the per-channel chain (test infrastructure only).

The same chain as `OracleChannel` / `or_channel_process` (extract -> FM
discriminator with the cross-block bridge -> stereo decode with pilot PLL,
lock hysteresis and mono fallback -> RDS baseband; or AM / SSB / CW), with
every intermediate in float64: no complex64 products, no float32 stores, an
exact NCO phase.  The algorithm's own constants stay as the reference defines
them, including the float32-valued extraction taps (the reference casts its
float64 LowpassFIR design to float32, gpudemod/stream_state.go:63-71, so those
values are part of the filter) and the FreqShift phase accumulated by repeated
float64 addition (dsp/freqshift.go:13-15).  The errors of the reference-
precision restatement and of the GPU against this truth are what the parity
report states per output.

Sources, step by step: streaming_host_core.go:5-64 (extraction: phase before
increment, the first T taps of the T|1 design, history of T-1),
demod/fm.go:179-196 and recorder/streamer.go:1287-1302 (discriminator and
bridge), recorder/streamer.go:1496-1644 and 1355-1404 (stereo decode, PLL,
lock, hysteresis, 15 kHz mono fallback), demod/fm.go:143-163, 234-271
(RDS baseband), demod/am.go:11-27, ssb.go:19-39, cw.go:11-26.
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np

from . import oracle as O

MODE_IQ, MODE_NFM, MODE_WFM, MODE_WFM_STEREO, MODE_AM, MODE_USB, MODE_LSB, MODE_CW = range(8)
TWO_PI = 2.0 * math.pi


class _FIR:
    """Stateful real FIR (dsp/fir_stateful.go): float64 delay line."""

    def __init__(self, taps):
        self.t = np.asarray(taps, dtype=np.float64)
        self.h = np.zeros(self.t.size - 1)

    def __call__(self, x):
        x = np.asarray(x, dtype=np.float64)
        w = np.concatenate([self.h, x])
        y = np.convolve(w, self.t)[self.t.size - 1:self.t.size - 1 + x.size]
        self.h = w[w.size - (self.t.size - 1):]
        return y


class Truth64Channel:
    def __init__(self, sample_rate, offset_hz, bandwidth, out_rate, num_taps, mode, rds=True):
        self.fs = int(sample_rate)
        self.D = O.exact_integer_decimation(sample_rate, out_rate)
        self.out_rate = int(out_rate)
        self.T = int(num_taps) if num_taps > 0 else 101
        self.h = O.base_taps_f32(bandwidth, sample_rate, self.T)[: self.T].astype(np.float64)
        self.mode = mode
        self.rds_on = rds
        self.offset = Fraction(offset_hz).limit_denominator(1 << 20)
        self.i0 = 0                      # stream index of the next input sample
        self.pc = 0                      # phase count
        self.hist = np.zeros(0, np.complex128)
        self.last = None
        # stereo state (streamer.go:1546-1555)
        r = self.out_rate
        lp = lambda c: O.lowpass_fir(c, r, 101)
        self.f_lpr, self.f_lrl = _FIR(lp(15000)), _FIR(lp(15000))
        self.f_bhi, self.f_blo = _FIR(lp(53000)), _FIR(lp(23000))
        self.f_phi, self.f_plo = _FIR(lp(21000)), _FIR(lp(17000))
        self.f_mono = _FIR(lp(15000))
        self.phase, self.freq = 0.0, TWO_PI * 19000 / r
        self.alpha, self.beta = O.pll_coefficients(50, 0.707, r)
        self.lpa = 1 - math.exp(-TWO_PI * 200 / r)
        self.I = self.Q = 0.0
        self.err_avg = 0.0
        self.on = self.off = 0
        self.enabled = False
        # RDS stream (fm.go:234-271 over the concatenated discriminator stream)
        self.rds_taps = O.lowpass_fir(7500, r, 101)
        self.rds_dr = max(1, r // 19000)
        self.rds_phase = 0.0
        self.rds_inc = -TWO_PI * (-57000.0) / r
        self.rds_count = 0
        self.rds_hist = np.zeros(0, np.complex128)

    # -- extraction -------------------------------------------------------
    def _extract(self, x):
        n = x.size
        # exact phase -2 pi frac(i * offset / fs) of stream sample i (phase
        # before increment), offset = num/den: integer arithmetic modulo den*fs
        num, den = self.offset.numerator, self.offset.denominator
        M = den * self.fs
        ii = np.arange(self.i0, self.i0 + n, dtype=np.int64)
        if abs(num) * (self.i0 + n) < (1 << 62):
            r = (ii * num) % M
        else:
            r = np.array([(int(i) * num) % M for i in ii], dtype=np.int64)
        fr_f = ((-r) % M).astype(np.float64) / M
        s = x.astype(np.complex128) * np.exp(1j * TWO_PI * fr_f)
        w = np.concatenate([self.hist, s])
        H = self.hist.size
        first = self.D - self.pc - 1           # newest sample of output 0 within the block
        nj = np.arange(first, n, self.D)
        out = np.zeros(nj.size, np.complex128)
        wpad = np.concatenate([np.zeros(self.T, np.complex128), w])
        for k in range(self.T):
            out += self.h[k] * wpad[self.T + H + nj - k]
        self.pc = (self.pc + n) % self.D
        keep = self.T - 1
        self.hist = w[max(0, w.size - keep):]
        self.i0 += n
        return out

    # -- stereo -----------------------------------------------------------
    def _stereo(self, d):
        n = d.size
        lpr = self.f_lpr(d)
        bpf = self.f_bhi(d) - self.f_blo(d)
        pil = self.f_phi(d) - self.f_plo(d)
        r = self.out_rate
        fmin, fmax = TWO_PI * 17000 / r, TWO_PI * 21000 / r
        ph, fq, I, Q = self.phase, self.freq, self.I, self.Q
        a, b, lpa = self.alpha, self.beta, self.lpa
        lr = np.empty(n)
        pp = es = 0.0
        for i in range(n):
            p = float(pil[i])
            I += lpa * (p * math.cos(ph) - I)
            Q += lpa * (-p * math.sin(ph) - Q)
            e = math.atan2(Q, I)
            fq += b * e
            fq = fmin if fq < fmin else (fmax if fq > fmax else fq)
            ph += fq + a * e
            if ph > TWO_PI:
                ph -= TWO_PI
            elif ph < 0:
                ph += TWO_PI
            pp += p * p
            es += abs(e)
            lr[i] = bpf[i] * 2 * math.sin(2 * ph)
        self.phase, self.freq, self.I, self.Q = ph, fq, I, Q
        self.err_avg = 0.9 * self.err_avg + 0.1 * (es / n)
        lr = self.f_lrl(lr)
        coh = (I * I + Q * Q) * n / pp if pp > 1e-12 else 0.0
        fhz = fq * r / TWO_PI
        locked = coh > 0.15 and abs(fhz - 19000) < 250 and self.err_avg < 0.35
        if locked:
            self.on += 1
            self.off = 0
            if self.on >= 4:
                self.enabled = True
        else:
            self.on = 0
            self.off += 1
            if self.off >= 10:
                self.enabled = False
        out = np.empty(2 * n)
        if self.enabled:
            out[0::2] = 0.5 * (lpr + lr)
            out[1::2] = 0.5 * (lpr - lr)
        else:
            m = self.f_mono(d)
            out[0::2] = m
            out[1::2] = m
        return out, locked

    def _rds(self, d):
        n = d.size
        # the reference adds inc one sample at a time (never wrapped)
        acc = np.empty(n)
        p = self.rds_phase
        for i in range(n):
            p += self.rds_inc
            acc[i] = p
        self.rds_phase = p
        c = d * np.exp(1j * acc)
        w = np.concatenate([self.rds_hist, c])
        H = self.rds_hist.size
        gi = self.rds_count + np.arange(n)
        keep = np.nonzero(gi % self.rds_dr == 0)[0]
        out = np.zeros(keep.size, np.complex128)
        for k in range(101):
            src = H + keep - k
            valid = (gi[keep] - k) >= 0
            out += np.where(valid, self.rds_taps[k] * w[np.clip(src, 0, None)], 0)
        self.rds_hist = w[max(0, w.size - 100):]
        self.rds_count += n
        return out

    def process(self, x):
        iq = self._extract(np.asarray(x))
        res = {"iq": iq, "audio": np.zeros(0), "rds": np.zeros(0, np.complex128), "locked": False, "stereo": False}
        m = self.mode
        if m in (MODE_NFM, MODE_WFM, MODE_WFM_STEREO):
            seq = iq if self.last is None else np.concatenate([[self.last], iq])
            if iq.size:
                self.last = iq[-1]
            d = np.angle(seq[1:] * np.conj(seq[:-1])) if seq.size >= 2 else np.zeros(0)
            if d.size:
                if m == MODE_NFM:
                    res["audio"] = d
                elif m == MODE_WFM:
                    res["audio"] = self.f_mono(d)
                else:
                    res["audio"], res["locked"] = self._stereo(d)
                    res["stereo"] = self.enabled
                if self.rds_on and m != MODE_NFM:
                    res["rds"] = self._rds(d)
        elif m == MODE_AM and iq.size:
            a = np.abs(iq)
            res["audio"] = a - a.mean()
        elif m in (MODE_USB, MODE_LSB, MODE_CW) and iq.size:
            bfo = -700.0 if m == MODE_LSB else 700.0
            ph = TWO_PI * bfo / self.out_rate * np.arange(1, iq.size + 1)
            if m == MODE_CW:
                res["audio"] = iq.real * np.cos(ph)
            else:
                res["audio"] = iq.real * np.cos(ph) - iq.imag * np.sin(ph)
        return res
