"""The learned search's threshold count, line by line (a model of the rule in
csrc/bt_learned.cu, on the CPU): a query counts the code line of its
predicted unit first and continues into the neighbouring lines only while the
count can continue there.  The result must equal the count over the whole
window, ua + #{j in [ua, ub): T_j <= q}, for windows of any width."""
import numpy as np

LINE = 59  # thresholds per code line


def count_line(T, line, q):
    j0 = line * LINE
    return int(np.count_nonzero(T[j0:j0 + LINE] <= q))


def window_part(ua, ub, j0, c):
    return max(0, min(ub, j0 + c) - max(ua, j0))


def line_by_line(T, ua, ub, pu, q):
    """(unit, code lines read) as the kernel's fresh pass and queue do it."""
    has = ub > ua
    pu = min(max(pu, ua), ub - 1 if has else ua)
    line = pu // LINE
    j0 = line * LINE
    la, lb = ua // LINE, ((ub - 1) // LINE if has else ua // LINE)
    c = count_line(T, line, q) if has else 0
    skip = window_part(ua, ub, j0, c)
    need = right = False
    if has:
        if c == 0 and la < line:
            need = True
        else:
            if la < line:
                skip += j0 - ua
            if lb > line and c >= LINE:
                need = right = True
    lines = 1
    while need:  # the queue passes
        line = line + 1 if right else line - 1
        lines += 1
        j0 = line * LINE
        c = count_line(T, line, q)
        skip += window_part(ua, ub, j0, c)
        if right:
            need = line < lb and c >= LINE
        else:
            need = line > la and c == 0
            if line > la and c > 0:
                skip += j0 - ua
    return ua + skip, lines


def test_line_by_line_count_equals_the_window_count():
    g = np.random.default_rng(1)
    for _ in range(3000):
        units = int(g.integers(1, 600))
        T = np.sort(g.integers(0, 1 << 20, size=units - 1))  # thresholds j < units - 1
        q = int(g.integers(-3, (1 << 20) + 3))
        ua = int(g.integers(0, units))
        ub = max(ua, min(units - 1, ua + int(g.integers(0, 240))))
        pu = int(g.integers(max(0, ua - 5), ub + 6))
        got, lines = line_by_line(T, ua, ub, pu, q)
        assert got == ua + int(np.count_nonzero(T[ua:ub] <= q))
        # never more lines than the window spans
        assert lines <= max(1, (ub - 1) // LINE - ua // LINE + 1)


def test_a_window_inside_one_line_reads_one_line():
    T = np.arange(0, 590 * 10, 10)
    for q in (-1, 0, 5, 155, 5895, 10 ** 6):
        got, lines = line_by_line(T, 60, 100, 80, q)
        assert lines == 1
        assert got == 60 + int(np.count_nonzero(T[60:100] <= q))
