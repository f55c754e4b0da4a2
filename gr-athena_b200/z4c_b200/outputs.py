"""Output files of the Z4c path in the reference's formats, so that scripts
written for the reference's output read these unchanged.

  HistoryOutput   HistoryOutput::WriteOutputFile (outputs/history.cpp:
                  370-445) for the Z4c columns: time, dt, N_MeshBlock and the
                  eight constraint norms of Z4c.hst_norms()
  TrackerOutput   PunctureTracker::WriteTracker (z4c/puncture_tracker.cpp:
                  36-80, 188-203): iteration, time, position and the shift
                  interpolated there
The psi4 multipole files are written by WaveExtract.Write.
"""
import os

Z4C_HST_COLUMNS = ("H-norm2", "M-norm2", "Mx-norm2", "My-norm2", "Mz-norm2", "Z-norm2",
                   "Theta-norm2", "C-norm2")


class HistoryOutput:
    """A `<problem_id>.hst` history file: the header is written when the file
    is new, then one row per call; `data_format` is the <output> block's
    data_format (default %12.5e), each value preceded by a blank."""

    def __init__(self, path, data_format="%12.5e", version="z4c_b200"):
        self.path = path
        self.fmt = " " + data_format
        self.version = version

    def write(self, time, dt, nblocks, norms):
        norms = list(norms)
        assert len(norms) == len(Z4C_HST_COLUMNS)
        new = not os.path.exists(self.path)
        with open(self.path, "a") as f:
            if new:
                f.write(f"# GR-Athena++ ({self.version}) history data\n")
                cols = ["time", "dt", "N_MeshBlock", *Z4C_HST_COLUMNS]
                f.write("# " + "".join(f"[{i + 1}]={c} " for i, c in enumerate(cols)) + "\n")
            row = self.fmt % time + self.fmt % dt + " %d" % int(nblocks)
            row += "".join(self.fmt % v for v in norms)
            f.write(row + "\n")


class TrackerOutput:
    """A puncture tracker file `<problem_id>.<filename><n>.txt` (filename
    from <z4c> filename, default "puncture_")."""

    def __init__(self, problem_id, n, filename="puncture_", directory="."):
        self.path = os.path.join(directory, f"{problem_id}.{filename}{n}.txt")

    def write(self, iteration, time, pos, beta):
        new = not os.path.exists(self.path)
        with open(self.path, "a") as f:
            if new:
                f.write("# 1:iter 2:time 3:x 4:y 5:z 6:betax 7:betay 8:betaz\n")
            f.write("%d %.15e %.15e %.15e %.15e %.15e %.15e %.15e\n"
                    % (int(iteration), time, *[float(v) for v in pos],
                       *[float(v) for v in beta]))
