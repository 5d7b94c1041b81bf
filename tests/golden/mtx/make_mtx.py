"""Writes the MatrixMarket fixtures of tests/test_mtx.py (small hand-made files covering
the formats the reader accepts).  Run from anywhere: python tests/golden/mtx/make_mtx.py"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))

FILES = {
    # general real, comments, a duplicate entry (summed), an empty line, unsorted entries
    "general.mtx": "%%MatrixMarket matrix coordinate real general\n"
                   "% a comment\n%another\n"
                   "4 5 7\n"
                   "3 2 -1.5\n1 1 2.0\n4 5 1e-3\n\n2 3 0.25\n1 4 -7\n3 2 0.5\n2 2 3.0\n",
    # symmetric: off-diagonal entries mirrored
    "symmetric.mtx": "%%MatrixMarket matrix coordinate real symmetric\n"
                     "3 3 4\n1 1 4\n2 1 -1\n3 2 -1\n3 3 4\n",
    # skew-symmetric: mirrored entries negated
    "skew.mtx": "%%MatrixMarket matrix coordinate real skew-symmetric\n"
                "3 3 2\n2 1 1.5\n3 1 -2\n",
    # pattern: every entry is 1.0
    "pattern.mtx": "%%MatrixMarket matrix coordinate pattern symmetric\n"
                   "3 3 3\n1 1\n2 1\n3 3\n",
    # integer field, upper-case banner words, CRLF line ends
    "integer.mtx": "%%MatrixMarket MATRIX Coordinate INTEGER General\r\n"
                   "2 2 3\r\n1 1 5\r\n2 1 -3\r\n2 2 7\r\n",
    # more entries in the file than the header announces: reading stops at the count
    "truncated.mtx": "%%MatrixMarket matrix coordinate real general\n"
                     "2 2 2\n1 1 1\n2 2 2\n1 2 99\n",
    # vectors
    "vec_array.mtx": "%%MatrixMarket matrix array real general\n% rhs\n4 1\n1.0\n-2.5\n3e2\n0.125\n",
    "vec_coord.mtx": "%%MatrixMarket matrix coordinate real general\n5\n2 1.5\n5 -3\n",
    "vec_nobanner.mtx": "first line is skipped\n3\n1 1\n3 9\n",
    # errors
    "complex.mtx": "%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n",
    "nobanner.mtx": "3 3 1\n1 1 1\n",
}

if __name__ == "__main__":
    for name, text in FILES.items():
        with open(os.path.join(HERE, name), "w", newline="") as f:
            f.write(text)
    print(f"wrote {len(FILES)} files to {HERE}")
