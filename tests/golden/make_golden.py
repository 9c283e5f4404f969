"""Copy the reference's golden recordings used by the parity tests into tests/golden/.

Run with the reference checkout given as an argument or in TE_REFERENCE:
    python tests/golden/make_golden.py REF
Copies, unchanged:
  data/kernels/kernels.json        kernel parameter ABI (binding index, ptr/ref, write)
and for each of the scenarios single_cell (120x120x40), squall_line (300x60x40, periodic
in y) and supercell_stretched (144x144x40, stretched grid):
  data/<scen>/tape.json            recorded command stream of steps 1-2
  data/<scen>/state/<id>.bin.gz    every buffer before step 1
  data/<scen>/hashes.ref.bin       per-dispatch region hashes of step 1
  data/<scen>/step1.json           FNV-1a of every buffer after step 1
These are recordings of the upstream implementation shipped with the reference
(web/view.js:1039-1068, web/replay.html:190-232); the tests replay them.
"""
import os
import shutil
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('TE_REFERENCE', '')
OUT = os.path.dirname(os.path.abspath(__file__))


SCENARIOS = ('single_cell', 'squall_line', 'supercell_stretched')


def main():
    if not REF or not os.path.isdir(os.path.join(REF, 'data')):
        sys.exit('usage: make_golden.py REF (the reference checkout; or set TE_REFERENCE)')
    shutil.copy(os.path.join(REF, 'data/kernels/kernels.json'), os.path.join(OUT, 'kernels.json'))
    for scen in SCENARIOS:
        src = os.path.join(REF, 'data', scen)
        dst = os.path.join(OUT, scen)
        os.makedirs(os.path.join(dst, 'state'), exist_ok=True)
        for f in ('tape.json', 'hashes.ref.bin', 'step1.json'):
            shutil.copy(os.path.join(src, f), os.path.join(dst, f))
        for f in os.listdir(os.path.join(src, 'state')):
            shutil.copy(os.path.join(src, 'state', f), os.path.join(dst, 'state', f))
    print('golden fixtures written to', OUT)


if __name__ == '__main__':
    main()
