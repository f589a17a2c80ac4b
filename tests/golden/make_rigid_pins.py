"""Extracts the values the reference's own rigid-body tests pin into JSON
fixtures: tests/block-sliding.py:64-80 (position x and velocity v_x of the
block at given callback indices, 1e-3 relative tolerance) into
block_sliding_ref.json, and tests/projectile.py:47-50 (the x distance in
inches at the end, 0.5% relative tolerance) into projectile_ref.json. Run with
the environment variable REFERENCE set to the reference source tree; the
tests read only the JSON."""
import ast
import json
import os
import re
import sys

REFERENCE = os.environ.get('REFERENCE')


def main():
    if not REFERENCE or not os.path.isdir(REFERENCE):
        sys.exit('set REFERENCE to the reference source tree')
    src = open(os.path.join(REFERENCE, 'tests', 'block-sliding.py')).read()
    m = re.search(r'REF\s*=\s*(\[[^\]]*\])', src)  # the test is Python 2: read the list literal alone
    if not m:
        sys.exit('REF list not found')
    values = ast.literal_eval(m.group(1))
    out = dict(source='tests/block-sliding.py of the reference (REF list)', tolerance=1e-3,
               step=1e-3, stop=10.0, friction=0.8, gravity=9.81,
               pins=[dict(quantity='x' if k == 0 else 'vx', index=int(i), value=float(v)) for k, i, v in values])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'block_sliding_ref.json')
    with open(path, 'w') as f:
        json.dump(out, f, indent=1)
    print(path, len(values), 'pins')
    src = open(os.path.join(REFERENCE, 'tests', 'projectile.py')).read()
    exact = float(re.search(r'exact\s*=\s*([0-9.eE+-]+)', src).group(1))
    tol = float(re.search(r'if \(error < ([0-9.eE+-]+)\)', src).group(1))
    out = dict(source='tests/projectile.py of the reference (exact, error bound)', quantity='x distance [in]',
               value=exact, tolerance=tol)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'projectile_ref.json')
    with open(path, 'w') as f:
        json.dump(out, f, indent=1)
    print(path, exact, tol)


if __name__ == '__main__':
    main()
