"""Regenerates the golden fixtures in this folder from the reference's own test
inputs (tan/tests/src/TALibTestConvolution/*.wav). Run here, where the
reference is mounted; the outputs are committed and nothing reads the
reference at test time.

    python tests/golden/make_golden.py REFERENCE_ROOT

Samples are converted short -> float as the reference's WAV reader does
(s / 32768, tan/common/wav.cpp:235).
"""
import json
import os
import sys
import wave

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = None  # set by main() from the required REFERENCE_ROOT argument


def read_wav(name):
    with wave.open(os.path.join(SRC, name)) as w:
        n, ch, sw, fs = w.getnframes(), w.getnchannels(), w.getsampwidth(), w.getframerate()
        assert sw == 2
        data = np.frombuffer(w.readframes(n), dtype="<i2").reshape(n, ch).T.copy()
    return data, fs


def main():
    global SRC
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py REFERENCE_ROOT")
    SRC = os.path.join(sys.argv[1], "tan/tests/src/TALibTestConvolution")
    resp, fs = read_wav("testresponse.wav")
    taps = []
    for c in range(resp.shape[0]):
        nz = np.nonzero(resp[c])[0]
        taps.append([{"index": int(i), "short": int(resp[c, i]), "value": float(resp[c, i]) / 32768.0} for i in nz])
    with open(os.path.join(HERE, "testresponse_taps.json"), "w") as f:
        json.dump({"source": "tan/tests/src/TALibTestConvolution/testresponse.wav", "rate": fs,
                   "length": int(resp.shape[1]), "channels": taps}, f, indent=1)

    pulses, _ = read_wav("pulsetrainS.wav")
    np.save(os.path.join(HERE, "pulsetrainS_head.npy"), pulses[:, :16384])

    dense, _ = read_wav("testresponse2.wav")
    np.save(os.path.join(HERE, "testresponse2_head.npy"), dense[:, :4096])
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
