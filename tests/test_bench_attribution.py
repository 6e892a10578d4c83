"""The benchmark's work attribution follows the runner's extraction choices:
the FM band's 40 stations are one tensor-core channel group (outputs 256..,
three TF32 passes of a 128 x 80 x 512 GEMM per tile), classes of fewer than
four channels, float64-summed FM channels and short-arm classes stay on the
FP32 forms, and the split keeps the total extraction work."""
import bench as B


def test_fm_band_is_one_group():
    chans = B.fm_band_channels()
    grouped, tflop = B.gemm_grouped(chans)
    assert grouped == set(range(40))
    tiles = -(-(B.BLOCK // 32 - 256) // 128)
    assert tflop == 3 * 2 * 128 * 80 * 2 * 8 * 32 * tiles
    w = B.algorithmic_work(chans)
    assert abs(w["extract_dense"]["flop"] + w["extract_gemm"]["flop"] - w["extract"]["flop"]) < 1e-3 * w["extract"]["flop"]
    assert w["extract_gemm"]["tensor_flop"] == tflop


def test_small_precise_and_short_arm_classes_are_not_grouped():
    few = [dict(kind="WFM", T=256, D=32, out_rate=312_500) for _ in range(3)]
    assert B.gemm_grouped(few)[0] == set()
    precise = [dict(kind="NFM", T=320, D=40, out_rate=250_000, bw=50_000.0) for _ in range(8)]
    assert B.gemm_grouped(precise)[0] == set()
    short_arm = [dict(kind="NFM", T=512, D=400, out_rate=25_000, bw=12_500.0) for _ in range(8)]
    assert B.extraction_form(512, 400) == "extract_mod"
    assert B.gemm_grouped(short_arm)[0] == set()
    odd = [dict(kind="WFM", T=250, D=25, out_rate=400_000) for _ in range(8)]
    assert B.gemm_grouped(odd)[0] == set()
